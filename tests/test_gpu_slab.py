"""The slab decomposition along x on one GPU: S slab handles stepped with
the x exchanges between them (device copies) against the single periodic
domain on the same state.  Fields and particles agree to round-off: a slab
holds positions in its own coordinates (x shifted by an integer, as each
rank of the reference does), so positions round differently from the
single domain's by a few ulps a step; currents sum in atomic order."""
import numpy as np
import pytest

from ._util import grid_and_config, random_fields, random_particles, to_gpu_fields, to_gpu_particles

pytestmark = pytest.mark.gpu


def _sorted(p, lens):
    """Live particles in a canonical order; a position within 1e-6 of the
    upper periodic edge is taken at the lower one (a particle on the edge may
    have wrapped in one run and not in the other)."""
    m = np.asarray(p.flv) != 0
    out = {k: np.asarray(getattr(p, k))[m].copy() for k in ("q", "x", "y", "z", "u", "v", "w", "flv")}
    for k, L in zip(("x", "y", "z"), lens):
        if L:
            out[k][out[k] > 3.0 + L - 1e-6] -= L
    o = np.lexsort((np.round(out["z"], 9), np.round(out["y"], 9), np.round(out["x"], 9), out["flv"]))
    return {k: v[o] for k, v in out.items()}


@pytest.mark.parametrize("dims,fdtd,nslabs,queued,fixed", [(3, "yee", 2, False, False), (3, "lehe", 3, True, False),
                                                            (2, "yee", 3, False, False), (2, "lehe", 2, True, False),
                                                            (3, "yee", 1, True, False), (3, "yee", 2, False, True),
                                                            (2, "lehe", 3, True, True), (3, "yee", 1, True, True)])
def test_slabs_track_single_domain(dims, fdtd, nslabs, queued, fixed):
    """6 steps (a reorder at step 3) of a 24-cell-wide domain as one
    periodic domain and as 1, 2 or 3 slabs (the library's phase calls
    waiting for their work, or queued with the exchanges ordered on the
    streams), particles up to 0.8 per momentum component, a fifth of them
    next to a face: the same live particles (positions and momenta to
    1e-11), E and B to 1e-11 of their scale."""
    import torch

    from pictor_b200 import Simulation
    from pictor_b200.slab import join_interior, join_particles, local_domain, split_fields, split_particles

    nx, ny, nz = 24, 8, 8
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, fdtd=fdtd, capacity=1 << 15, reorder_period=3)
    f = to_gpu_fields(random_fields(g, seed=71, scale=0.05))
    p = to_gpu_particles(random_particles(g, n=6000, seed=72, umax=0.8))
    with Simulation(cfg) as s:
        s.load_particles(p)
        s.load_fields(f)
        s.step(6)
        assert s.device_errors() == 0
        ref_p, ref_f = s.fetch_particles(), s.fetch_fields(with_current=False)
    dom = local_domain(cfg, nslabs, device=torch.device("cuda", 0), out_capacity=4096, queued=queued, fixed=fixed)
    try:
        for sl, ps, fs in zip(dom.slabs, split_particles(p, nx, nslabs), split_fields(f, nx, nslabs)):
            sl.sim.load_particles(ps)
            sl.sim.load_fields(fs)
        dom.step(6)
        for sl in dom.slabs:
            assert sl.sim.device_errors() == 0
        got_p = join_particles([sl.sim.fetch_particles() for sl in dom.slabs], nx)
        got_f = [sl.sim.fetch_fields(with_current=False) for sl in dom.slabs]
    finally:
        dom.close()
    lens = (nx, ny, nz if dims == 3 else 0)
    a, b = _sorted(got_p, lens), _sorted(ref_p, lens)
    assert len(a["x"]) == len(b["x"])
    np.testing.assert_array_equal(a["flv"], b["flv"])
    np.testing.assert_array_equal(a["q"], b["q"])
    for k, L in zip(("x", "y", "z"), lens):
        d = a[k] - b[k]
        if L:
            d -= L * np.round(d / L)     # the same point on the periodic axis
        assert np.abs(d).max() <= 1e-11, k
    for k in ("u", "v", "w"):
        np.testing.assert_allclose(a[k], b[k], rtol=0, atol=1e-11, err_msg=k)
    for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        ref = getattr(ref_f, n)[2:-3]
        got = join_interior(got_f, n)
        if dims == 3:
            ref, got = ref[:, 2:-3, 2:-3], got[:, 2:-3, 2:-3]
        else:
            ref, got = ref[:, 2:-3, :], got[:, 2:-3, :]
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-11 * max(np.abs(ref).max(), 1e-30), err_msg=n)


def test_slab_refuses_the_periodic_entry_points():
    """A slab's step has exchanges between its phases: pic_step and the
    single-domain particle exchange refuse it; the slab form is Cartesian
    without a current filter."""
    from pictor_b200 import PicError, Simulation

    g, cfg = grid_and_config(dims=2, nx=12, ny=8)
    cfg.slab_x = 1
    with Simulation(cfg) as s:
        with pytest.raises(PicError):
            s.step(1)
        with pytest.raises(PicError):
            s.exchange_particles()
    for bad in (dict(curr_filter=1),):
        g, cfg = grid_and_config(dims=2, nx=12, ny=8, **bad)
        cfg.slab_x = 1
        with pytest.raises(PicError):
            Simulation(cfg)


@pytest.mark.parametrize("dims,nslabs,fixed", [(3, 2, False), (2, 3, False), (3, 2, True)])
def test_fp32_slabs_track_single_domain(dims, nslabs, fixed):
    """The FP32 cell-relative form split into slabs: its mover leaves an x
    leaver in the ghost cell beside the face, the pack sends it in the
    8-double layout (x in the receiver's coordinates) and leaves a hole, the
    receiver appends it converted back, and after a reorder the tiled mover
    moves the bricks while the particles received since then are moved one
    per thread.  6 steps (reorders at 3 and 6) against the FP32 single
    periodic domain: the same live particles, positions to 1e-5 of a cell
    and momenta to 1e-5 (the FP32 currents sum in a different order), E and
    B to 1e-5 of their scale."""
    import torch

    from pictor_b200 import Simulation
    from pictor_b200.slab import join_interior, join_particles, local_domain, split_fields, split_particles

    nx, ny, nz = 24, 8, 8
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, precision="fp32", capacity=1 << 15, reorder_period=3)
    f = to_gpu_fields(random_fields(g, seed=73, scale=0.05))
    p = to_gpu_particles(random_particles(g, n=6000, seed=74, umax=0.8, holes=0.0))
    with Simulation(cfg) as s:
        s.load_particles(p)
        s.load_fields(f)
        s.step(6)
        assert s.device_errors() == 0
        ref_p, ref_f = s.fetch_particles(), s.fetch_fields(with_current=False)
    dom = local_domain(cfg, nslabs, device=torch.device("cuda", 0), out_capacity=4096, fixed=fixed)
    try:
        for sl, ps, fs in zip(dom.slabs, split_particles(p, nx, nslabs), split_fields(f, nx, nslabs)):
            sl.sim.load_particles(ps)
            sl.sim.load_fields(fs)
        dom.step(6)
        for sl in dom.slabs:
            assert sl.sim.device_errors() == 0
        got_p = join_particles([sl.sim.fetch_particles() for sl in dom.slabs], nx)
        got_f = [sl.sim.fetch_fields(with_current=False) for sl in dom.slabs]
    finally:
        dom.close()
    lens = (nx, ny, nz if dims == 3 else 0)
    a, b = _sorted(got_p, lens), _sorted(ref_p, lens)
    assert len(a["x"]) == len(b["x"]) == 6000
    np.testing.assert_array_equal(a["flv"], b["flv"])
    for k, L in zip(("x", "y", "z"), lens):
        d = a[k] - b[k]
        if L:
            d -= L * np.round(d / L)
        assert np.abs(d).max() <= 1e-5, (k, np.abs(d).max())
    for k in ("u", "v", "w"):
        np.testing.assert_allclose(a[k], b[k], rtol=0, atol=1e-5, err_msg=k)
    for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        ref = getattr(ref_f, n)[2:-3]
        got = join_interior(got_f, n)
        if dims == 3:
            ref, got = ref[:, 2:-3, 2:-3], got[:, 2:-3, 2:-3]
        else:
            ref, got = ref[:, 2:-3], got[:, 2:-3]
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-5 * max(np.abs(ref).max(), 1e-30), err_msg=n)


@pytest.mark.parametrize("nslabs,fixed", [(2, False), (3, False), (3, True)])
def test_cylindrical_slabs_track_single_domain(nslabs, fixed):
    """The FP64 cylindrical step split along r: slab 0 holds the axis (the
    near-axis sub-steps, the axis field and current conditions), the last
    slab's high face is the outer radius, the faces between them are
    exchanged; 6 steps with a reorder at step 3 (the tiled mover after it)
    of r-weighted electrons and ions with a few particles crossing the axis
    region equal the single domain's: the same live particles (positions and
    momenta to 1e-11), E and B to 1e-11 of their scale."""
    import torch

    from oracle import oracle as O
    from pictor_b200 import PicConfig, Simulation
    from pictor_b200.slab import join_interior, join_particles, local_domain, split_fields, split_particles

    nx, ny, nz = 24, 8, 10
    cfg = PicConfig(nx=nx, ny=ny, nz=nz, dims=3, c=0.45, qi=0.01, qm=(1.0, -1.0), geom="cylindrical",
                    capacity=1 << 15, reorder_period=3, rmin=-0.5, inc_axis=1)
    g = O.make_grid(3, nx, ny, nz, c=0.45, qi=0.01, qm=(1.0, -1.0))
    op = O.cyl_load_uniform(g, 1, 1, 1, 1.0, 2e-3, -1.0, 2, 5, 1 << 14)
    rng = np.random.default_rng(5)
    idx = rng.choice(op.used, 60, replace=False)
    op.x[idx] = 3.5 + rng.uniform(0.05, 1.0, 60)          # near the axis, moving through it
    op.u[idx] = rng.uniform(-0.6, 0.6, 60)
    op.v[idx] = rng.uniform(-0.6, 0.6, 60)
    out_idx = rng.choice(op.used, 200, replace=False)       # some fast radial movers near the slab faces
    op.u[out_idx] = rng.uniform(-0.9, 0.9, 200)
    op.flv[idx[:30]] = 1
    op.q[idx[:30]] *= -1.0
    p = to_gpu_particles(op)
    f = to_gpu_fields(random_fields(g, seed=73, scale=0.02))
    with Simulation(cfg) as s:
        s.load_particles(p)
        s.load_fields(f)
        s.step(6)
        assert s.device_errors() == 0
        ref_p, ref_f = s.fetch_particles(), s.fetch_fields(with_current=False)
    dom = local_domain(cfg, nslabs, device=torch.device("cuda", 0), out_capacity=4096, fixed=fixed)
    try:
        for sl, ps, fs in zip(dom.slabs, split_particles(p, nx, nslabs), split_fields(f, nx, nslabs)):
            sl.sim.load_particles(ps)
            sl.sim.load_fields(fs)
        dom.step(6)
        for sl in dom.slabs:
            assert sl.sim.device_errors() == 0
        got_p = join_particles([sl.sim.fetch_particles() for sl in dom.slabs], nx)
        got_f = [sl.sim.fetch_fields(with_current=False) for sl in dom.slabs]
    finally:
        dom.close()
    lens = (0, ny, nz)          # r is not periodic
    a, b = _sorted(got_p, lens), _sorted(ref_p, lens)
    assert len(a["x"]) == len(b["x"])
    np.testing.assert_array_equal(a["flv"], b["flv"])
    np.testing.assert_array_equal(a["q"], b["q"])
    for k, L in zip(("x", "y", "z"), lens):
        d = a[k] - b[k]
        if L:
            d -= L * np.round(d / L)
        assert np.abs(d).max() <= 1e-11, k
    for k in ("u", "v", "w"):
        np.testing.assert_allclose(a[k], b[k], rtol=0, atol=1e-11, err_msg=k)
    for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        ref = getattr(ref_f, n)[2:-3][:, 2:-3, 2:-3]
        got = join_interior(got_f, n)[:, 2:-3, 2:-3]
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-11 * max(np.abs(ref).max(), 1e-30), err_msg=n)


def test_fixed_boxes_overflow_moves_nothing():
    """Fixed-size boxes too small for the particles leaving a slab: the pack
    moves nothing (both counts 0, the leavers stay where the mover left
    them) and returns PIC_ERR_OVERFLOW."""
    import torch

    from pictor_b200 import PicError
    from pictor_b200.slab import local_domain, split_fields, split_particles

    nx, ny, nz = 24, 8, 8
    g, cfg = grid_and_config(dims=3, nx=nx, ny=ny, nz=nz, capacity=1 << 15)
    p = to_gpu_particles(random_particles(g, n=6000, seed=74, umax=0.8))
    f = to_gpu_fields(random_fields(g, seed=75, scale=0.05))
    dom = local_domain(cfg, 2, device=torch.device("cuda", 0), out_capacity=2, fixed=True)
    try:
        for sl, ps, fs in zip(dom.slabs, split_particles(p, nx, 2), split_fields(f, nx, 2)):
            sl.sim.load_particles(ps)
            sl.sim.load_fields(fs)
        sl = dom.slabs[0]
        n0 = sl.sim.particle_count()
        sl.sim.update_b_half()
        sl.sim.move_deposit()
        with pytest.raises(PicError) as e:
            sl.pack_particles_fixed()
        assert e.value.code == -3                           # PIC_ERR_OVERFLOW
        tl, tr, _, _ = sl.boxes()
        assert tl[0].item() == 0.0 and tr[0].item() == 0.0
        assert sl.sim.particle_count() == n0
    finally:
        dom.close()
