"""Field faces of EnforceBC_Final (src/bc/bc.F90:292-340) on the GPU
against the oracle: 'attn' faces (Attenuate_EM_Vacuum), an 'iflw' face with
a uniform flow (Attenuate_EM_Flow) and 'open' x faces (OpenBC_Fld_Left /
Right), each bit-exact on random fields (the same FP64 operations per
component), then 'attn' faces on x and y in a 10-step lockstep with
particles, called where MAIN.F90 calls EnforceBC_Final (after AddCurrent)."""
import numpy as np
import pytest

from oracle import oracle as O

from ._util import grid_and_config, random_fields, to_gpu_fields, to_gpu_particles

pytestmark = pytest.mark.gpu

NAMES6 = ("Ex", "Ey", "Ez", "Bx", "By", "Bz")


def _compare(gf, of, exact=True, tol=0.0):
    for n in NAMES6:
        a, b = getattr(gf, n), getattr(of, n)
        if exact:
            np.testing.assert_array_equal(a, b, err_msg=n)
        else:
            np.testing.assert_allclose(a, b, rtol=0, atol=tol * max(np.abs(b).max(), 1e-30), err_msg=n)


@pytest.mark.parametrize("dims", [2, 3])
def test_field_faces_exact(dims):
    from pictor_b200 import Simulation

    nx, ny, nz = (24, 16, 1) if dims == 2 else (14, 12, 10)
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz)
    faces = {1: (2.3, 4.0), 2: (nx - 3.5, 3.0), 3: (1.7, 4.0), 4: (ny - 2.0, 2.5)}
    if dims == 3:
        faces.update({5: (1.5, 4.0), 6: (nz - 2.5, 4.0)})
    cases = [
        ("vacuum", faces),
        ("vacuum", {2: (nx - 4.0, 4.0)}),
        ("flow", (2, nx - 3.0, 2.0, 4.0, (0.01, -0.02, 0.1), (-0.3, 0.05, 0.0))),
        ("flow", (3, 2.0, 1.0, 4.0, (0.0, 0.05, 0.0), (0.0, 0.2, 0.1))),
        ("open", (1, nx - 5.2)),
        ("open", (0, 2.0)),
    ]
    for kind, arg in cases:
        f = random_fields(g, seed=hash((kind, str(arg))) % 1000, consistent_ghosts=False)
        o = O.Oracle(g, O.Particles(1), f.copy())
        with Simulation(cfg) as s:
            s.load_fields(to_gpu_fields(f))
            if kind == "vacuum":
                o.attenuate_vacuum(arg)
                s.Attenuate_EM_Vacuum(arg)
            elif kind == "flow":
                side, pos, dl, sc, b, v = arg
                o.attenuate_flow(side, pos, dl, sc, b, v)
                s.Attenuate_EM_Flow(side, pos, dl, sc, b, v)
            else:
                o.open_fld_x(*arg)
                s.OpenBC_Fld_x(*arg)
            _compare(s.fetch_fields(), o.f)


def test_field_faces_invalid():
    from pictor_b200 import PicError, Simulation

    g, cfg = grid_and_config(dims=2, nx=16, ny=12)
    with Simulation(cfg) as s:
        for call in (lambda: s.Attenuate_EM_Vacuum({5: (1.0, 4.0)}),       # z face in 2D
                     lambda: s.Attenuate_EM_Vacuum({1: (1.0, 0.0)}),       # scale 0
                     lambda: s.Attenuate_EM_Flow(5, 3.0),                  # face 5 has no flow layer
                     lambda: s.OpenBC_Fld_x(2, 3.0)):
            with pytest.raises(PicError) as e:
                call()
            assert e.value.code == -1


@pytest.mark.parametrize("dims", [2, 3])
def test_attenuating_faces_lockstep(dims):
    from pictor_b200 import Simulation

    nx, ny, nz = (32, 16, 1) if dims == 2 else (16, 12, 8)
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, reorder_period=5, qi=0.00158203125, capacity=1 << 17)
    faces = {1: (3.0, 4.0), 2: (nx - 4.0, 4.0), 4: (ny - 3.0, 3.0)}
    p = O.load_weibel(dims, nx, ny, nz, epc=4 if dims == 3 else 8, drift=0.5, temp=0.01, seed=23)
    o = O.Oracle(g, p.copy())
    with Simulation(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        for t in range(1, 11):
            o.update_b_half(); o.send_recv_flds("B"); s.update_b_half()
            o.move_deposit(); s.move_deposit()
            o.exchange_particles(); s.exchange_particles()
            o.update_b_half(); o.send_recv_flds("B"); s.update_b_half()
            o.update_e(); o.send_recv_flds("E"); s.update_e()
            o.fold_current(); s.fold_current()
            o.add_current(); o.send_recv_flds("E"); s.add_current()
            o.attenuate_vacuum(faces); s.Attenuate_EM_Vacuum(faces)
            if t % 5 == 0:
                o.reorder(); s.reorder()
        assert s.device_errors() == 0
        gf = s.fetch_fields(with_current=False)
        gp = s.fetch_particles()
    v = o.p.view()
    assert np.array_equal(gp.flv, v["flv"])
    for k in ("x", "y", "z", "u", "v", "w"):
        np.testing.assert_allclose(getattr(gp, k), v[k], rtol=1e-9, atol=1e-9, err_msg=k)
    _compare(gf, o.f, exact=False, tol=1e-9)
    # beyond the upper x face by more than its scale every component is gone
    assert not gf.Ey[nx + 2:].any()


def _particles_close(gp, op, u_rtol):
    v = op.view()
    assert len(gp.x) == op.used
    assert np.array_equal(gp.flv, v["flv"])
    for k in ("q", "x", "y", "z", "v", "w"):
        np.testing.assert_array_equal(getattr(gp, k), v[k], err_msg=k)
    np.testing.assert_allclose(gp.u, v["u"], rtol=u_rtol, atol=0, err_msg="u")


@pytest.mark.parametrize("dims", [2, 3])
def test_open_faces_lockstep(dims):
    """'open' faces on both x sides for fields and particles, called after
    AddCurrent as EnforceBC_Final orders them (fields, then the right and
    the left particle face), 8 steps with a reorder every 4: after the first
    call the particle arrays equal the oracle's slot for slot (holes and the
    appended copies in the same order; the copies' u to 1e-14, the column
    means being FP64 atomic sums), thereafter to 1e-9."""
    from pictor_b200 import Simulation

    nx, ny, nz = (32, 16, 1) if dims == 2 else (16, 12, 8)
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, reorder_period=4, qi=0.00158203125, capacity=1 << 18)
    p = O.load_weibel(dims, nx, ny, nz, epc=4 if dims == 3 else 8, drift=0.5, temp=0.01, seed=29)
    pl, pr = 2.0, nx - 3.0
    o = O.Oracle(g, p.copy())
    with Simulation(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        for t in range(1, 9):
            o.update_b_half(); o.send_recv_flds("B"); s.update_b_half()
            o.move_deposit(); s.move_deposit()
            o.exchange_particles(); s.exchange_particles()
            o.update_b_half(); o.send_recv_flds("B"); s.update_b_half()
            o.update_e(); o.send_recv_flds("E"); s.update_e()
            o.fold_current(); s.fold_current()
            o.add_current(); o.send_recv_flds("E"); s.add_current()
            o.open_fld_x(0, pl); s.OpenBC_Fld_x(0, pl)
            o.open_fld_x(1, pr); s.OpenBC_Fld_x(1, pr)
            assert o.open_prtl_x(1, pr) == 0; s.OpenBC_Prtl_x(1, pr)
            assert o.open_prtl_x(0, pl) == 0; s.OpenBC_Prtl_x(0, pl)
            if t == 1:
                assert o.p.used > len(p.view()["x"])            # copies were appended
                _particles_close(s.fetch_particles(), o.p, 1e-14)
            if t % 4 == 0:
                o.reorder(); s.reorder()
        assert s.device_errors() == 0
        gf = s.fetch_fields(with_current=False)
        gp = s.fetch_particles()
    v = o.p.view()
    assert np.array_equal(gp.flv, v["flv"])
    for k in ("x", "y", "z", "u", "v", "w"):
        np.testing.assert_allclose(getattr(gp, k), v[k], rtol=1e-9, atol=1e-9, err_msg=k)
    _compare(gf, o.f, exact=False, tol=1e-9)
    live = v["flv"] != 0
    assert (v["x"][live] > pl + 3 - 1).all() and (v["x"][live] < pr + 3 + 1).all()


def test_open_particle_face_overflow():
    """Copies that do not fit in the capacity: PIC_ERR_OVERFLOW with the
    error word's OVERFLOW bit, nothing appended (the count stays), the
    particles beyond the face made holes as the oracle makes them."""
    from pictor_b200 import PicError, Simulation

    nx, ny = 24, 12
    g, cfg = grid_and_config(dims=2, nx=nx, ny=ny)
    p = O.load_weibel(2, nx, ny, 1, epc=8, drift=0.3, temp=0.01, seed=31)
    n = p.used
    cfg.capacity = n + 8                                    # far fewer free slots than the layer's particles
    o = O.Oracle(g, p.copy())
    o.p.capacity = n + 8
    assert o.open_prtl_x(1, nx - 4.0) == -1
    with Simulation(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        with pytest.raises(PicError) as e:
            s.OpenBC_Prtl_x(1, nx - 4.0)
        assert e.value.code == -3                           # PIC_ERR_OVERFLOW
        assert s.device_errors() & 2
        assert s.particle_count() == n
        gp = s.fetch_particles()
    v = o.p.view()
    assert np.array_equal(gp.flv, v["flv"]) and (v["flv"] == 0).sum() > (p.view()["flv"] == 0).sum()
