"""Error statuses of the C ABI, each one made on the host: a capacity that
is too small, a particle with a non-finite momentum, a particle outside the
ghost frame.  These are the reference's Abort(12) paths
(src/mem/particles_gpu.F90:21, src/comm/communication.F90:96-102); here the
kernels set a bit of the handle's error word and skip the access, the call
returns the PIC_ERR_* code, and the handle stays usable.  No case faults or
hangs the GPU: every index a kernel forms from particle data is checked
before the access it guards."""
import numpy as np
import pytest

from ._util import grid_and_config, random_fields, random_particles, to_gpu_fields, to_gpu_particles

pytestmark = pytest.mark.gpu

DEVERR_RANGE, DEVERR_OVERFLOW, DEVERR_NAN = 1, 2, 4


def _code(fn):
    from pictor_b200 import PicError

    with pytest.raises(PicError) as e:
        fn()
    return e.value.code


def _leaving(dims, n=3000):
    """Particles a fifth of which sit next to a face and move fast enough to
    leave through it, with the fields that push them."""
    g, cfg = grid_and_config(dims=dims, nx=16, ny=12, nz=10, capacity=n)
    p = random_particles(g, n=n, seed=5, umax=2.0, near_boundary=0.5, holes=0.0)
    f = random_fields(g, seed=6, scale=0.05)
    return g, cfg, p, f


@pytest.mark.parametrize("dims", [2, 3])
def test_wrap_past_capacity_returns_overflow(dims):
    """capacity == live particles: the wrap has no slot to append a leaver
    to (AppendParticles past gpu_prtl_arr_size).  Nothing is moved, the
    count stays, the error word holds OVERFLOW; after the word is cleared
    the handle works again."""
    from pictor_b200 import Simulation

    g, cfg, p, f = _leaving(dims)
    with Simulation(cfg) as s:
        s.load_fields(to_gpu_fields(f))
        s.load_particles(to_gpu_particles(p))
        s.move_deposit()
        before = s.fetch_particles()
        assert _code(s.exchange_particles) == -3   # PIC_ERR_OVERFLOW
        assert s.particle_count() == p.used
        assert s.device_errors() & DEVERR_OVERFLOW
        after = s.fetch_particles()
        for k in ("q", "x", "y", "z", "u", "v", "w", "flv"):
            assert np.array_equal(getattr(after, k), getattr(before, k)), k
        # the full step (one CUDA graph) reports it the same way
        assert _code(lambda: s.step(1)) == -3
        assert s.device_errors() & DEVERR_OVERFLOW
        assert s.device_errors() == 0


def test_loader_past_capacity_returns_overflow():
    """The Weibel loader makes more particles than the capacity holds."""
    from pictor_b200 import Simulation

    for prec in ("fp64", "fp32"):
        g, cfg = grid_and_config(dims=2, nx=16, ny=12, precision=prec, capacity=100)
        with Simulation(cfg) as s:
            assert _code(lambda: s.init_weibel(8, 0.5, 0.5, 0.005, 0.005, 2930)) == -3
            assert s.device_errors() & DEVERR_OVERFLOW


@pytest.mark.parametrize("prec,dims", [("fp64", 2), ("fp64", 3), ("fp32", 2), ("fp32", 3)])
def test_non_finite_momentum_returns_nan(prec, dims):
    """One particle with a NaN momentum and one with an infinite one: the
    mover raises NAN and no index is formed from a non-finite position.  The
    FP64 movers leave both particles where they were; the FP32 mover keeps
    their cells (their offsets turn NaN); the other particles move."""
    from pictor_b200 import Simulation

    g, cfg = grid_and_config(dims=dims, nx=16, ny=12, nz=10, precision=prec, capacity=1 << 14)
    p = random_particles(g, n=2000, seed=8, umax=0.5, holes=0.0)
    gp = to_gpu_particles(p)
    gp.u[10] = np.nan
    gp.w[20] = np.inf
    with Simulation(cfg) as s:
        s.load_particles(gp)
        x0 = s.fetch_particles().x.copy()
        assert _code(s.move_deposit) == -4   # PIC_ERR_NAN
        assert s.device_errors() & DEVERR_NAN
        got = s.fetch_particles()
        # both forms fetch in slot order, which no reorder has changed
        for i in (10, 20):
            if prec == "fp64":
                assert got.x[i] == x0[i]
            else:
                assert np.isnan(got.x[i]) or np.floor(got.x[i]) == np.floor(x0[i])
        moved = np.abs(got.x - x0) > 0
        assert moved.sum() > 1500
        if prec == "fp64":   # the FP32 particles' NaN current reaches J, as it would in the reference
            assert np.isfinite(s.fetch_fields().Jx).all()


@pytest.mark.parametrize("dims", [2, 3])
def test_particle_outside_the_ghost_frame_returns_range(dims):
    """A particle at x = 1.5 (the ghost frame starts at 2): the FP64 mover
    raises RANGE and skips it; the FP32 form refuses it at the load."""
    from pictor_b200 import Simulation

    g, cfg = grid_and_config(dims=dims, nx=16, ny=12, nz=10, capacity=1 << 14)
    p = random_particles(g, n=500, seed=9, holes=0.0)
    gp = to_gpu_particles(p)
    gp.x[7] = 1.5
    with Simulation(cfg) as s:
        s.load_particles(gp)
        assert _code(s.move_deposit) == -7   # PIC_ERR_RANGE
        assert s.device_errors() & DEVERR_RANGE
        assert s.fetch_particles().x[7] == 1.5
    g, cfg = grid_and_config(dims=dims, nx=16, ny=12, nz=10, precision="fp32", capacity=1 << 14)
    with Simulation(cfg) as s:
        assert _code(lambda: s.load_particles(gp)) == -7
        assert s.device_errors() & DEVERR_RANGE


def test_slab_outbox_overflow():
    """A slab whose outbox holds 4 particles while far more leave through
    its x faces: pic_slab_pack_particles returns OVERFLOW with both counts
    zero and the particle count unchanged, in the queued mode too."""
    import ctypes as C

    import torch

    from pictor_b200.slab import P_WORDS, Slab

    g, cfg, p, f = _leaving(2, n=3000)
    cfg.capacity = 1 << 14
    for queued in (False, True):
        sl = Slab(cfg, 0, 1, device=torch.device("cuda", 0), out_capacity=4)
        try:
            s = sl.sim
            s.load_particles(to_gpu_particles(p))
            s.load_fields(to_gpu_fields(f))
            s.set_sync(not queued)
            s.move_deposit()
            nr, nl = C.c_int64(-1), C.c_int64(-1)
            rc = s.L.pic_slab_pack_particles(s.h, sl.out.data_ptr(), 4, C.byref(nr), C.byref(nl))
            assert rc == -3
            assert nr.value == 0 and nl.value == 0
            assert s.device_errors() & DEVERR_OVERFLOW
            s.set_sync(True)
            assert s.particle_count() == p.used
            assert sl.out.numel() == P_WORDS * 4
        finally:
            sl.close()
