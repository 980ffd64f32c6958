"""Particle injection at an 'iflw' face (InjectNewPrtl, src/bc/bc_inflow.F90:
134-256) on the GPU against the oracle: the same Philox draws, so the same
trials are accepted and the particles are appended in the same order with
positions bit for bit and momenta to 1e-13 (the device's sqrt, cos and sin
against libm's); every face in 2D and the z faces in 3D, the Poisson count
of a small region, a moving injector; then 10 steps of a plasma flowing in
through the upper x face while the lower x face removes what reaches it,
injection called after the move as EnforceBC_PostMovDep calls it; and the
capacity overflow."""
import numpy as np
import pytest

from oracle import oracle as O

from ._util import assert_particles_equal, grid_and_config, to_gpu_particles

pytestmark = pytest.mark.gpu

SP = [(1, 2e-3, 1.0), (2, 8e-3, -1.0)]


def _close(gp, op):
    v = op.view()
    assert len(gp.x) == op.used
    assert np.array_equal(gp.flv, v["flv"])
    for k in ("q", "x", "y", "z"):
        np.testing.assert_array_equal(getattr(gp, k), v[k], err_msg=k)
    for k in ("u", "v", "w"):
        np.testing.assert_allclose(getattr(gp, k), v[k], rtol=1e-13, atol=1e-15, err_msg=k)


@pytest.mark.parametrize("dims,face,pos,drift,speed,epc", [
    (2, 1, 6.0, (0.3, 0.0, 0.0), 0.0, 400.0),
    (2, 2, 26.0, (-0.3, 0.1, 0.0), 0.0, 400.0),
    (2, 3, 4.0, (0.0, 0.4, 0.0), 0.5, 400.0),
    (2, 4, 14.0, (0.05, -0.2, 0.0), 0.0, 6.0),        # a small region: the Poisson count
    (3, 5, 3.0, (0.0, 0.0, 0.3), 0.0, 200.0),
    (3, 6, 9.0, (0.1, 0.0, -0.3), 0.2, 200.0),
])
def test_injection_matches_oracle(dims, face, pos, drift, speed, epc):
    from pictor_b200 import Simulation

    nx, ny, nz = (32, 18, 1) if dims == 2 else (14, 12, 12)
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, capacity=1 << 17)
    o = O.Oracle(g, O.Particles(1 << 17))
    o.p.used = 0
    with Simulation(cfg) as s:
        for call in (0, 1):
            n = o.inject(face, pos, SP, epc=epc, density=0.8, drift=drift, speed=speed, vmax=0.8, seed=5, call=call)
            s.InflowBC_Prtl(face, pos, SP, epc=epc, density=0.8, drift=drift, speed=speed, vmax=0.8, seed=5, call=call)
            assert n > 0
            assert s.particle_count() == o.p.used
        _close(s.fetch_particles(), o.p)
        assert s.device_errors() == 0


def test_inflow_lockstep():
    from pictor_b200 import Simulation

    nx, ny = 32, 16
    g, cfg = grid_and_config(dims=2, nx=nx, ny=ny, reorder_period=5, qi=0.00158203125, capacity=1 << 17)
    p = O.load_weibel(2, nx, ny, 1, epc=4, drift=0.2, temp=0.01, seed=71)
    o = O.Oracle(g, p.copy())
    pos = nx - 2.0
    flow = (-0.3, 0.0, 0.0)
    with Simulation(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        for t in range(1, 11):
            o.update_b_half(); o.send_recv_flds("B"); s.update_b_half()
            o.move_deposit(); s.move_deposit()
            o.inject(2, pos, SP, epc=8.0, density=1.0, drift=flow, vmax=0.5, seed=3, call=t)
            s.InflowBC_Prtl(2, pos, SP, epc=8.0, density=1.0, drift=flow, vmax=0.5, seed=3, call=t)
            o.remove_particles(1, 1.0); s.RemovePrtl(1, 1.0)
            o.exchange_particles(); s.exchange_particles()
            if t == 1:
                _close(s.fetch_particles(), o.p)
            o.update_b_half(); o.send_recv_flds("B"); s.update_b_half()
            o.update_e(); o.send_recv_flds("E"); s.update_e()
            o.fold_current(); s.fold_current()
            o.add_current(); o.send_recv_flds("E"); s.add_current()
            if t % 5 == 0:
                o.reorder(); s.reorder()
        assert s.device_errors() == 0
        gp = s.fetch_particles()
        gf = s.fetch_fields(with_current=False)
    v = o.p.view()
    assert np.array_equal(gp.flv, v["flv"])
    for k in ("x", "y", "z", "u", "v", "w"):
        np.testing.assert_allclose(getattr(gp, k), v[k], rtol=1e-9, atol=1e-9, err_msg=k)
    for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        a, b = getattr(gf, n), getattr(o.f, n)
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-9 * max(np.abs(b).max(), 1e-30), err_msg=n)


@pytest.mark.parametrize("dims", [2, 3])
def test_fluid_frame_reflection_matches_oracle(dims):
    """RefPrtlFluidFrameRight on the GPU against the oracle for random
    particles and fields-free J: the reflected particles bit for bit, J to
    1e-12 of its scale (FP64 atomics against the serial sum)."""
    from pictor_b200 import Simulation

    from ._util import random_particles

    nx, ny, nz = (32, 16, 1) if dims == 2 else (16, 12, 10)
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz)
    p = random_particles(g, n=8000, seed=81, umax=0.5, near_boundary=0.0)
    pos = nx - 6.0
    o = O.Oracle(g, p.copy())
    with Simulation(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        o.reflect_fluid_right(pos, -0.3)
        s.RefPrtlFluidFrameRight(pos, -0.3)
        assert_particles_equal(s.fetch_particles(), o.p, exact=True)
        f = s.fetch_fields()
        for n in ("Jx", "Jy", "Jz"):
            a, b = getattr(f, n), getattr(o.f, n)
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * max(np.abs(b).max(), 1e-30), err_msg=n)
        assert np.abs(o.f.Jx).max() > 0
        assert s.device_errors() == 0


def test_injection_past_capacity():
    from pictor_b200 import PicError, Simulation

    g, cfg = grid_and_config(dims=2, nx=32, ny=16, capacity=1000)
    with Simulation(cfg) as s:
        with pytest.raises(PicError) as e:
            s.InflowBC_Prtl(2, 20.0, SP, epc=4000.0, density=1.0, drift=(-0.3, 0.0, 0.0), vmax=0.5, seed=1, call=0)
        assert e.value.code == -3
        assert s.device_errors() & 2
        assert s.particle_count() == 0
