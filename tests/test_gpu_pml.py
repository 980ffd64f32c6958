"""The convolutional PML (src/bc/bc_pml.F90) on the GPU against the oracle:
UpdateMagFld_PML and UpdateElcFld_PML, each followed by the halo, bit for
bit on random fields over repeated calls (the psi grids carry over), 2D and
3D; the FP64 form in a 10-step lockstep with particles and PML faces on both
x sides, the calls where MAIN.F90 makes them (after the second B half step
and after the E update); and a plane pulse leaving the box through the
layers, in the FP64 and the FP32 forms."""
import numpy as np
import pytest

from oracle import oracle as O

from ._util import grid_and_config, random_fields, to_gpu_fields, to_gpu_particles

pytestmark = pytest.mark.gpu

NAMES6 = ("Ex", "Ey", "Ez", "Bx", "By", "Bz")

CASES = [
    (2, (30, 14, 1), {1: (4.0, 3.0), 2: (23.5, 4.0)}),
    (2, (24, 20, 1), {3: (2.2, 4.0), 4: (15.0, 2.0), 2: (18.0, 4.0)}),
    (3, (16, 12, 10), {1: (3.0, 2.5), 2: (11.0, 4.0), 5: (2.0, 3.0), 6: (6.5, 2.0)}),
    (3, (12, 16, 8), {3: (3.5, 4.0), 4: (12.0, 3.0)}),
]


@pytest.mark.parametrize("dims,n,faces", CASES)
def test_pml_exact(dims, n, faces):
    from pictor_b200 import Simulation

    g, cfg = grid_and_config(dims=dims, nx=n[0], ny=n[1], nz=n[2])
    f = random_fields(g, seed=41 + dims, consistent_ghosts=False)
    o = O.Oracle(g, O.Particles(1), f.copy())
    pml = O.Pml(g, faces)
    with Simulation(cfg) as s:
        s.load_fields(to_gpu_fields(f))
        s.SetBC_PML(faces)
        for _ in range(3):
            o.pml_b(pml); o.send_recv_flds("B"); s.UpdateMagFld_PML()
            o.pml_e(pml); o.send_recv_flds("E"); s.UpdateElcFld_PML()
        gf = s.fetch_fields(with_current=False)
    for k in NAMES6:
        np.testing.assert_array_equal(getattr(gf, k), getattr(o.f, k), err_msg=k)


@pytest.mark.parametrize("dims", [2, 3])
def test_pml_lockstep(dims):
    from pictor_b200 import Simulation

    nx, ny, nz = (32, 16, 1) if dims == 2 else (16, 12, 8)
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, reorder_period=5, qi=0.00158203125, capacity=1 << 17)
    faces = {1: (4.0, 3.0), 2: (nx - 5.0, 3.0)}
    p = O.load_weibel(dims, nx, ny, nz, epc=4 if dims == 3 else 8, drift=0.5, temp=0.01, seed=37)
    o = O.Oracle(g, p.copy())
    pml = O.Pml(g, faces)
    with Simulation(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        s.SetBC_PML(faces)
        for t in range(1, 11):
            o.update_b_half(); o.send_recv_flds("B"); s.update_b_half()
            o.move_deposit(); s.move_deposit()
            o.exchange_particles(); s.exchange_particles()
            o.update_b_half(); o.pml_b(pml); o.send_recv_flds("B")
            s.update_b_half(); s.UpdateMagFld_PML()
            o.update_e(); o.pml_e(pml); o.send_recv_flds("E")
            s.update_e(); s.UpdateElcFld_PML()
            o.fold_current(); s.fold_current()
            o.add_current(); o.send_recv_flds("E"); s.add_current()
            if t % 5 == 0:
                o.reorder(); s.reorder()
        assert s.device_errors() == 0
        gf = s.fetch_fields(with_current=False)
        gp = s.fetch_particles()
    v = o.p.view()
    assert np.array_equal(gp.flv, v["flv"])
    for k in ("x", "y", "z", "u", "v", "w"):
        np.testing.assert_allclose(getattr(gp, k), v[k], rtol=1e-9, atol=1e-9, err_msg=k)
    for k in NAMES6:
        a, b = getattr(gf, k), getattr(o.f, k)
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-9 * max(np.abs(b).max(), 1e-30), err_msg=k)
    assert np.abs(o.f.Ez).max() > 0


def _pulse(precision: str, steps: int):
    """The energy left of a plane Ez/By pulse moving along +x in vacuum after
    `steps` field steps, with PML faces on both x sides."""
    from pictor_b200 import Simulation

    nx, ny = 96, 8
    g, cfg = grid_and_config(dims=2, nx=nx, ny=ny, precision=precision, capacity=64)
    f = O.Fields(g)
    x = np.arange(g.mx) - 3.0
    f.Ez[...] = np.exp(-((x - 40.0) / 5.0) ** 2)[:, None, None]
    f.By[...] = -np.exp(-((x + 0.5 - 40.0) / 5.0) ** 2)[:, None, None]
    with Simulation(cfg) as s:
        s.load_fields(to_gpu_fields(f))
        s.SetBC_PML({1: (10.0, 8.0), 2: (85.0, 8.0)})
        d0 = s.diagnostics()
        out = []
        for t in range(1, steps + 1):
            s.update_b_half()
            s.update_b_half(); s.UpdateMagFld_PML()
            s.update_e(); s.UpdateElcFld_PML()
            if t % 60 == 0:
                d = s.diagnostics()
                out.append((d["E2"] + d["B2"]) / (d0["E2"] + d0["B2"]))
    return np.array(out)


def test_pml_absorbs_pulse_fp64_and_fp32():
    e64 = _pulse("fp64", 240)
    e32 = _pulse("fp32", 240)
    assert abs(e64[0] - 1.0) < 0.01            # the pulse has not reached the layers at step 60
    assert e64[-1] < 1e-3 and e32[-1] < 1e-3
    np.testing.assert_allclose(e32[:2], e64[:2], rtol=1e-5)


def test_pml_invalid():
    from pictor_b200 import PicError, Simulation

    g, cfg = grid_and_config(dims=2, nx=16, ny=12)
    with Simulation(cfg) as s:
        for faces in ({5: (1.0, 4.0)},          # z face in 2D
                      {1: (2.0, 0.0)}):         # thickness 0
            with pytest.raises(PicError) as e:
                s.SetBC_PML(faces)
            assert e.value.code == -1
        s.SetBC_PML({})                         # off: the phase calls do nothing
        s.UpdateMagFld_PML()
        s.UpdateElcFld_PML()
