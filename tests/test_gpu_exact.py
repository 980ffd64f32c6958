"""The FP64 form with the current summed in the reference's serial order
(pic_config.exact_current = 1): every phase of the step, the current
included, equals the serial CPU restatement bit for bit, so whole runs
agree bit for bit with it, and with themselves across a restart."""
import numpy as np
import pytest

from oracle import oracle as O

from ._util import grid_and_config, random_fields, random_particles, to_gpu_fields, to_gpu_particles

pytestmark = pytest.mark.gpu

CASES = [(2, "yee"), (2, "lehe"), (3, "yee"), (3, "lehe")]
NAMES = ("q", "x", "y", "z", "u", "v", "w")


def _sim(cfg):
    from pictor_b200 import Simulation

    return Simulation(cfg)


def _assert_state_equal(s, o, with_current=True):
    gp = s.fetch_particles()
    v = o.p.view()
    assert len(gp.x) == o.p.used
    for k in NAMES:
        bad = np.nonzero(getattr(gp, k) != v[k])[0]
        assert bad.size == 0, f"{k}: {bad.size} differ, first {bad[:4]}"
    assert np.array_equal(gp.flv, v["flv"])
    gf = s.fetch_fields(with_current=with_current)
    for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz") + (("Jx", "Jy", "Jz") if with_current else ()):
        assert np.array_equal(getattr(gf, n), getattr(o.f, n)), n


@pytest.mark.parametrize("dims", [2, 3])
def test_exact_current_of_one_move(dims):
    """One MoveDepositPrtl with the exact-order current: J equals the serial
    VecJ sums and ReduceCurrentMatrix scatter bit for bit."""
    g, cfg = grid_and_config(dims=dims, bext=(0.01, -0.02, 0.03))
    cfg.exact_current = 1
    f = random_fields(g, seed=21)
    p = random_particles(g, n=5000, seed=22)
    o = O.Oracle(g, p.copy(), f.copy())
    with _sim(cfg) as s:
        s.load_fields(to_gpu_fields(f))
        s.load_particles(to_gpu_particles(p))
        o.move_deposit()
        s.move_deposit()
        _assert_state_equal(s, o)


@pytest.mark.parametrize("dims,fdtd", CASES)
def test_exact_current_steps_bit_exact(dims, fdtd):
    """13 full steps (one CUDA graph each, reorders at 5 and 10) of the
    Weibel set-up: particles, E, B bit for bit after every step."""
    nx, ny, nz = (24, 20, 1) if dims == 2 else (12, 10, 8)
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, fdtd=fdtd, reorder_period=5,
                             qi=0.00158203125, capacity=1 << 17)
    cfg.exact_current = 1
    p = O.load_weibel(dims, nx, ny, nz, epc=4 if dims == 3 else 8, drift=0.5, temp=0.005, seed=7)
    o = O.Oracle(g, p.copy())
    with _sim(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        for t in range(1, 14):
            o.step(t, 5)
            s.step(1)
            if t in (1, 5, 6, 13):
                _assert_state_equal(s, o, with_current=False)


def test_restart_continues_bit_for_bit():
    """Run 7 steps, fetch the state (fields with ghosts, every particle slot,
    holes included, and the step counter, which fixes the reorder phase),
    destroy the handle; a new handle loaded from it runs 6 more steps.  The
    result equals 13 uninterrupted steps bit for bit (J is zero between
    steps, so it needs no transfer)."""
    from pictor_b200 import Particles

    nx, ny = 32, 24
    g, cfg = grid_and_config(dims=2, nx=nx, ny=ny, reorder_period=5, qi=0.00158203125, capacity=1 << 16)
    cfg.exact_current = 1
    p = O.load_weibel(2, nx, ny, epc=8, drift=0.5, temp=0.005, seed=12)
    with _sim(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        s.step(13)
        ref_p, ref_f = s.fetch_particles(), s.fetch_fields(with_current=False)
    with _sim(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        s.step(7)
        snap_p, snap_f = s.fetch_particles(), s.fetch_fields(with_current=False)
    with _sim(cfg) as s:
        s.load_particles(Particles(*(getattr(snap_p, k) for k in Particles.NAMES)))
        s.load_fields(snap_f)
        s.set_step(7)
        s.step(6)
        got_p, got_f = s.fetch_particles(), s.fetch_fields(with_current=False)
    for k in Particles.NAMES:
        assert np.array_equal(getattr(got_p, k), getattr(ref_p, k)), k
    for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        assert np.array_equal(getattr(got_f, n), getattr(ref_f, n)), n


def test_exact_current_is_reproducible():
    """Two runs of the same state give the same bits (the atomic form's
    current depends on the order the atomics land in)."""
    nx, ny, nz = 16, 12, 10
    g, cfg = grid_and_config(dims=3, nx=nx, ny=ny, nz=nz, reorder_period=4, qi=0.00158203125, capacity=1 << 16)
    cfg.exact_current = 1
    p = O.load_weibel(3, nx, ny, nz, epc=4, drift=0.5, temp=0.005, seed=13)
    out = []
    for _ in range(2):
        with _sim(cfg) as s:
            s.load_particles(to_gpu_particles(p))
            s.step(9)
            out.append(s.fetch_fields(with_current=False))
    for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        assert np.array_equal(getattr(out[0], n), getattr(out[1], n)), n


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_fetch_fields_into_caller_arrays(precision):
    """pic_fetch_fields into arrays the caller owns (here views of one
    reused buffer, as a host with pinned output buffers passes them) equals
    the fetch into fresh arrays; arrays of the wrong shape or order are
    refused before anything is written."""
    from pictor_b200 import Fields

    g, cfg = grid_and_config(dims=3, nx=12, ny=10, nz=8, precision=precision)
    f = random_fields(g, seed=77)
    shape = tuple(cfg.shape)
    n = int(np.prod(shape))
    buf = np.full(9 * n, np.nan)
    out = Fields(*(buf[c * n:(c + 1) * n].reshape(shape, order="F") for c in range(9)))
    with _sim(cfg) as s:
        s.load_fields(to_gpu_fields(f))
        ref = s.fetch_fields()
        got = s.fetch_fields(out=out)
        assert got is out
        bad = Fields(*(np.zeros(shape) for _ in range(9)))          # C order
        with pytest.raises(ValueError):
            s.fetch_fields(out=bad)
    for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Jx", "Jy", "Jz"):
        assert np.array_equal(getattr(out, k), getattr(ref, k)), k
