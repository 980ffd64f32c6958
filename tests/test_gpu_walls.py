"""Walls along x and y (src/bc/bc_reflect.F90 on one rank) on the GPU
against the oracle, phase by phase as MAIN.F90 calls them: reflecting
particle walls after the move (EnforceBC_PostMovDep) and conducting field
walls after AddCurrent (EnforceBC_Final), 10 steps with a reorder every 5."""
import numpy as np
import pytest

from oracle import oracle as O

from ._util import assert_particles_equal, grid_and_config, to_gpu_particles

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,fdtd,axis", [(2, "yee", "x"), (3, "lehe", "x"), (2, "lehe", "y"), (3, "yee", "y")])
def test_walls_lockstep(dims, fdtd, axis):
    from pictor_b200 import Simulation

    nx, ny, nz = (24, 16, 1) if dims == 2 else (12, 10, 8)
    n_ax = nx if axis == "x" else ny
    pl, pr = 1.5, n_ax - 2.5                    # walls at local 4.5 and n + 0.5 along the axis
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, fdtd=fdtd, reorder_period=5, qi=0.00158203125,
                             capacity=1 << 17)
    p = O.load_weibel(dims, nx, ny, nz, epc=4 if dims == 3 else 8, drift=0.6, temp=0.01, seed=17)
    o = O.Oracle(g, p.copy())
    with Simulation(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        for t in range(1, 11):
            o.update_b_half(); o.send_recv_flds("B"); s.update_b_half()
            o.move_deposit(); s.move_deposit()
            for side, pos in ((0, pl), (1, pr)):
                getattr(o, "reflect_particles_" + axis)(side, pos)
                getattr(s, "RefBC_Prtl_" + axis)(side, pos)
            o.exchange_particles(); s.exchange_particles()
            if t == 1:
                assert_particles_equal(s.fetch_particles(), o.p, exact=True)
                np.testing.assert_allclose(s.fetch_fields().Jx, o.f.Jx, rtol=0, atol=1e-12 * np.abs(o.f.Jx).max())
            o.update_b_half(); o.send_recv_flds("B"); s.update_b_half()
            o.update_e(); o.send_recv_flds("E"); s.update_e()
            o.fold_current(); s.fold_current()
            o.add_current(); o.send_recv_flds("E"); s.add_current()
            for side, pos in ((0, pl), (1, pr)):
                getattr(o, "conducting_" + axis)(side, pos)
                getattr(s, "CondBC_Fld_" + axis)(side, pos)
            if t % 5 == 0:
                o.reorder(); s.reorder()
        assert s.device_errors() == 0
        gp = s.fetch_particles()
        gf = s.fetch_fields(with_current=False)
    v = o.p.view()
    assert len(gp.x) == o.p.used
    live = v["flv"] != 0
    c = v[axis][live]
    assert ((c >= 4.5) & (c <= n_ax + 0.5)).all()                           # every particle between the walls
    assert np.array_equal(gp.flv, v["flv"])
    for k in ("x", "y", "z", "u", "v", "w"):
        np.testing.assert_allclose(getattr(gp, k), v[k], rtol=1e-9, atol=1e-9, err_msg=k)
    for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        a, b = getattr(gf, n), getattr(o.f, n)
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-9 * max(np.abs(b).max(), 1e-30), err_msg=n)
    if axis == "x":                                                          # tangential E beyond the low wall
        assert not gf.Ey[:4].any() and not gf.Ez[:4].any()
    else:
        assert not gf.Ex[:, :4].any() and not gf.Ez[:, :4].any()


@pytest.mark.parametrize("dims", [2, 3])
def test_remove_faces_lockstep(dims):
    """Particles removed beyond walls on the low x face and the high y face
    (and the low z face in 3D) every step, after the move: the same holes
    and the same survivors as the oracle, 8 steps with a reorder every 4."""
    from pictor_b200 import Simulation

    nx, ny, nz = (24, 16, 1) if dims == 2 else (12, 10, 8)
    faces = [(1, 2.5), (4, ny - 3.5)] + ([(5, 2.0)] if dims == 3 else [])
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, reorder_period=4, qi=0.00158203125, capacity=1 << 17)
    p = O.load_weibel(dims, nx, ny, nz, epc=4 if dims == 3 else 8, drift=0.6, temp=0.01, seed=23)
    o = O.Oracle(g, p.copy())
    with Simulation(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        for t in range(1, 9):
            o.update_b_half(); o.send_recv_flds("B"); s.update_b_half()
            o.move_deposit(); s.move_deposit()
            for face, pos in faces:
                o.remove_particles(face, pos)
                s.RemovePrtl(face, pos)
            o.exchange_particles(); s.exchange_particles()
            if t == 1:
                assert_particles_equal(s.fetch_particles(), o.p, exact=True)
            o.update_b_half(); o.send_recv_flds("B"); s.update_b_half()
            o.update_e(); o.send_recv_flds("E"); s.update_e()
            o.fold_current(); s.fold_current()
            o.add_current(); o.send_recv_flds("E"); s.add_current()
            if t % 4 == 0:
                o.reorder(); s.reorder()
        assert s.device_errors() == 0
        gp = s.fetch_particles()
    v = o.p.view()
    assert len(gp.x) == o.p.used < len(p.view()["x"])                      # holes dropped by the reorders
    assert np.array_equal(gp.flv, v["flv"])
    for k in ("x", "y", "z", "u", "v", "w", "q"):
        np.testing.assert_allclose(getattr(gp, k), v[k], rtol=1e-9, atol=1e-9, err_msg=k)
