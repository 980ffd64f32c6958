"""Parity of the CUDA path (through the C ABI) with the CPU restatement.

FP64 path: field updates, halo, fold, AddCurrent, the push, the wrap and the
reorder are bit-exact; J is compared at 1e-12 of its scale because the
deposit sums with atomics in a different order than the serial loop.
"""
import numpy as np
import pytest

from oracle import oracle as O

from ._util import (assert_particles_equal, grid_and_config, interior, random_fields, random_particles,
                    to_gpu_fields, to_gpu_particles)

pytestmark = pytest.mark.gpu

CASES = [(2, "yee"), (2, "lehe"), (3, "yee"), (3, "lehe")]


def _sim(cfg):
    from pictor_b200 import Simulation

    return Simulation(cfg)


@pytest.mark.parametrize("dims,fdtd", CASES)
def test_field_phases_bit_exact(dims, fdtd):
    g, cfg = grid_and_config(dims=dims, fdtd=fdtd)
    f = random_fields(g, seed=11)
    o = O.Oracle(g, O.Particles(1), f.copy())
    with _sim(cfg) as s:
        s.load_fields(to_gpu_fields(f))
        # B half step + halo (MAIN.F90:49-58)
        o.update_b_half(); o.send_recv_flds("B")
        s.update_b_half()
        gf = s.fetch_fields()
        for n in ("Bx", "By", "Bz", "Ex", "Ey", "Ez"):
            assert np.array_equal(getattr(gf, n), getattr(o.f, n)), n
        # E step + halo (MAIN.F90:108-110)
        o.update_e(); o.send_recv_flds("E")
        s.update_e()
        gf = s.fetch_fields()
        for n in ("Ex", "Ey", "Ez"):
            assert np.array_equal(getattr(gf, n), getattr(o.f, n)), n
        # current fold + AddCurrent + halo (MAIN.F90:124, 170-184)
        rng = np.random.default_rng(5)
        J = [np.asfortranarray(rng.normal(scale=1e-3, size=O.grid_shape(g))) for _ in range(3)]
        o.f.Jx[...], o.f.Jy[...], o.f.Jz[...] = J
        s.load_current(*J)
        o.fold_current()
        s.fold_current()
        gf = s.fetch_fields()
        for n in ("Jx", "Jy", "Jz"):
            assert np.array_equal(interior(getattr(gf, n), g), interior(getattr(o.f, n), g)), n
        o.add_current(); o.send_recv_flds("E")
        s.add_current()
        gf = s.fetch_fields()
        for n in ("Ex", "Ey", "Ez"):
            assert np.array_equal(getattr(gf, n), getattr(o.f, n)), n


@pytest.mark.parametrize("dims", [2, 3])
def test_move_deposit_parity(dims):
    g, cfg = grid_and_config(dims=dims, bext=(0.01, -0.02, 0.03))
    f = random_fields(g, seed=21)
    p = random_particles(g, n=5000, seed=22)
    o = O.Oracle(g, p.copy(), f.copy())
    with _sim(cfg) as s:
        s.load_fields(to_gpu_fields(f))
        s.load_particles(to_gpu_particles(p))
        o.move_deposit()
        s.move_deposit()
        gp = s.fetch_particles()
        assert_particles_equal(gp, o.p, exact=True)
        gf = s.fetch_fields()
        for n in ("Jx", "Jy", "Jz"):
            a, b = getattr(gf, n), getattr(o.f, n)
            scale = np.abs(b).max()
            assert scale > 0
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * scale, err_msg=n)


@pytest.mark.parametrize("dims", [2, 3])
def test_exchange_and_reorder_bit_exact(dims):
    g, cfg = grid_and_config(dims=dims)
    f = random_fields(g, seed=31, scale=0.2)
    p = random_particles(g, n=6000, seed=32, umax=2.0, near_boundary=0.5)
    o = O.Oracle(g, p.copy(), f.copy())
    with _sim(cfg) as s:
        s.load_fields(to_gpu_fields(f))
        s.load_particles(to_gpu_particles(p))
        o.move_deposit(); s.move_deposit()
        assert o.exchange_particles() == 0
        s.exchange_particles()
        assert s.particle_count() == o.p.used
        assert o.p.used > p.used, "test needs particles leaving through the faces"
        assert_particles_equal(s.fetch_particles(), o.p, exact=True)
        perm = o.reorder()
        s.reorder()
        assert s.particle_count() == o.p.used
        assert_particles_equal(s.fetch_particles(), o.p, exact=True)
        assert perm.size == o.p.used


@pytest.mark.parametrize("dims", [2, 3])
def test_tiled_f64_mover_after_reorder(dims):
    """After a reorder the FP64 mover runs by tiles of cells (node box and
    64-bit fixed-point current box in shared memory): positions and momenta
    bit-exact to the oracle, J to 1e-12 of its scale; three moves in a row
    (the boxes follow the particles' cells), wraps appending particles past
    the sorted range (moved per particle) in between."""
    g, cfg = grid_and_config(dims=dims, nx=40 if dims == 2 else 20, ny=24 if dims == 2 else 12,
                             nz=10, bext=(0.01, -0.02, 0.03))
    cfg.fp64_tiles = 1   # tiles on this small grid too
    f = random_fields(g, seed=41)
    p = random_particles(g, n=20000 if dims == 2 else 12000, seed=42, umax=1.5)
    # particles left in ghost cells (an edge leaver that the exchange sent
    # through one face only): the reorder sorts them into ghost-cell keys,
    # and a tile must still move them
    p.x[:3] = [2.6, g.mx - 1.6, 5.5]
    p.y[:3] = [4.2, 2.3, g.my - 1.7]
    o = O.Oracle(g, p.copy(), f.copy())
    with _sim(cfg) as s:
        s.load_fields(to_gpu_fields(f))
        s.load_particles(to_gpu_particles(p))
        o.reorder(); s.reorder()
        for it in range(3):
            o.move_deposit(); s.move_deposit()
            assert_particles_equal(s.fetch_particles(), o.p, exact=True)
            gf = s.fetch_fields()
            for n in ("Jx", "Jy", "Jz"):
                a, b = getattr(gf, n), getattr(o.f, n)
                np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * np.abs(b).max(), err_msg=n)
            o.exchange_particles(); s.exchange_particles()
            assert s.particle_count() == o.p.used
        assert s.device_errors() == 0


@pytest.mark.parametrize("tiles", [-1, 1])
@pytest.mark.parametrize("dims,fdtd", CASES)
def test_full_steps_lockstep(dims, fdtd, tiles):
    """Whole steps (one CUDA graph per step) against orc_step: identical
    particle state after the first step; thereafter the deposit's summation
    order enters E at round-off and the comparison uses tolerances.  The FP64
    mover per particle and by tiles (after the reorders at steps 5, 10)."""
    nx, ny, nz = (24, 20, 1) if dims == 2 else (12, 10, 8)
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, fdtd=fdtd, reorder_period=5,
                             qi=0.00158203125, capacity=1 << 17)
    cfg.fp64_tiles = tiles
    p = O.load_weibel(dims, nx, ny, nz, epc=4 if dims == 3 else 8, drift=0.5, temp=0.005, seed=7)
    o = O.Oracle(g, p.copy())
    with _sim(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        o.step(1, 5); s.step(1)
        assert_particles_equal(s.fetch_particles(), o.p, exact=True)
        for t in range(2, 13):
            o.step(t, 5); s.step(1)
        assert s.particle_count() == o.p.used
        gp = s.fetch_particles()
        v = o.p.view()
        assert np.array_equal(gp.flv, v["flv"])
        for k in ("x", "y", "z", "u", "v", "w"):
            np.testing.assert_allclose(getattr(gp, k), v[k], rtol=1e-9, atol=1e-9, err_msg=k)
        gf = s.fetch_fields(with_current=False)
        for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
            a, b = getattr(gf, n), getattr(o.f, n)
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-9 * max(np.abs(b).max(), 1e-30), err_msg=n)


@pytest.mark.parametrize("dims", [2, 3])
def test_weibel_loader_matches_oracle(dims):
    nx, ny, nz = (32, 24, 1) if dims == 2 else (12, 10, 8)
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, capacity=1 << 17)
    p = O.load_weibel(dims, nx, ny, nz, epc=8, drift=0.5, temp=0.005, seed=2930)
    with _sim(cfg) as s:
        n = s.init_weibel(8, 0.5, 0.5, 0.005, 0.005, 2930)
        assert n == p.used
        gp = s.fetch_particles()
        v = p.view()
        for k in ("x", "y", "z", "q"):
            assert np.array_equal(getattr(gp, k), v[k]), k
        assert np.array_equal(gp.flv, v["flv"])
        for k in ("u", "v", "w"):  # device cos/sin may differ from libm in the last bits
            np.testing.assert_allclose(getattr(gp, k), v[k], rtol=1e-13, atol=1e-15, err_msg=k)


@pytest.mark.parametrize("dims", [2, 3])
def test_gauss_residual_conserved_fp64(dims):
    nx, ny, nz = (32, 32, 1) if dims == 2 else (12, 12, 12)
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, qi=0.00158203125, capacity=1 << 18)
    with _sim(cfg) as s:
        s.init_weibel(16 if dims == 2 else 4, 0.5, 0.5, 0.005, 0.005, 2930)
        d0 = s.diagnostics()
        assert d0["gauss_linf"] <= 1e-14 * d0["rho_max"]
        s.step(40)
        d = s.diagnostics()
        # 2D zigzag conserves charge exactly; the reference's 3D weights leave an O(d^3) residual
        assert d["gauss_linf"] <= (1e-12 if dims == 2 else 1e-2) * d["rho_max"], d
        assert d["E2"] > 0 and d["B2"] > 0


def test_diagnostics_match_oracle():
    g, cfg = grid_and_config(dims=2, nx=24, ny=24, qi=0.00158203125)
    p = O.load_weibel(2, 24, 24, epc=8, drift=0.5, temp=0.005, seed=3)
    o = O.Oracle(g, p.copy())
    with _sim(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        for t in range(1, 6):
            o.step(t)
        s.step(5)
        eb, ee = o.field_energy()
        d = s.diagnostics()
        np.testing.assert_allclose([d["B2"], d["E2"]], [eb, ee], rtol=1e-9)
        res, rmax = o.gauss_residual()
        assert d["gauss_linf"] <= 1e-12 * rmax and res <= 1e-12 * rmax


@pytest.mark.parametrize("dims,prec", [(2, "fp64"), (3, "fp64"), (2, "fp32"), (3, "fp32")])
def test_kinetic_energy_matches_oracle(dims, prec):
    """CalcPrtlEnergy (savedata_routines.F90:283-308) per species on the
    device (FP64 accumulation) against orc_particle_energy, on the loader's
    particles and after 6 steps.  FP64: the sums differ by their order only
    (1e-12); FP32: the momenta are FP32 (1e-6 of each species' energy)."""
    nx, ny, nz = (24, 24, 1) if dims == 2 else (10, 8, 8)
    sc_qi = 0.00158203125
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, qi=sc_qi, precision=prec, reorder_period=4)
    p = O.load_weibel(dims, nx, ny, nz, epc=8, drift=0.5, temp=0.005, seed=4)
    o = O.Oracle(g, p.copy())
    masse = sc_qi
    tol = 1e-12 if prec == "fp64" else 1e-6
    with _sim(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        np.testing.assert_allclose(s.diagnostics(masse)["kinetic"], o.particle_energy(masse), rtol=tol)
        s.step(6)
        # the oracle's energies of the device's own particles after 6 steps
        o2 = O.Oracle(g, O.Particles.from_arrays(1 << 15, **{k: getattr(s.fetch_particles(), k)
                                                              for k in ("q", "x", "y", "z", "u", "v", "w", "flv")}))
        ke = s.diagnostics(masse)["kinetic"]
        assert (ke > 0).all()
        np.testing.assert_allclose(ke, o2.particle_energy(masse), rtol=tol if prec == "fp64" else 1e-9)


@pytest.mark.parametrize("dims", [2, 3])
def test_current_filter_bit_exact(dims):
    """smoothen_current (current.F90:19-163): two passes of the (1/4,1/2,1/4)
    filter on a folded current; interior bit-exact, then a filtered full step."""
    g, cfg = grid_and_config(dims=dims, curr_filter=2)
    rng = np.random.default_rng(8)
    J = [np.asfortranarray(rng.normal(scale=1e-3, size=O.grid_shape(g))) for _ in range(3)]
    o = O.Oracle(g, O.Particles(1))
    o.f.Jx[...], o.f.Jy[...], o.f.Jz[...] = J
    with _sim(cfg) as s:
        s.load_current(*J)
        o.fold_current(); s.fold_current()
        o.filter_current(2); s.filter_current()
        gf = s.fetch_fields()
        for n in ("Jx", "Jy", "Jz"):
            assert np.array_equal(interior(getattr(gf, n), g), interior(getattr(o.f, n), g)), n


def test_filtered_step_matches_oracle():
    g, cfg = grid_and_config(dims=2, nx=24, ny=20, curr_filter=1, qi=0.00158203125, reorder_period=5)
    p = O.load_weibel(2, 24, 20, epc=8, drift=0.5, temp=0.005, seed=5)
    o = O.Oracle(g, p.copy())
    with _sim(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        o.step_filtered(1, 5, 1); s.step(1)
        assert_particles_equal(s.fetch_particles(), o.p, exact=True)
        for t in range(2, 8):
            o.step_filtered(t, 5, 1); s.step(1)
        gf = s.fetch_fields(with_current=False)
        for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
            a, b = getattr(gf, n), getattr(o.f, n)
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-9 * max(np.abs(b).max(), 1e-30), err_msg=n)


def _fixed_point_slack(p, dims, nx, ny, nz, capacity, c, qi):
    """Bound of the tiled mover's fixed-point rounding in one J entry: each
    brick sums its current in units of 1/S, S = 2^30 / (c qi max|w| max(N, 256))
    for its N particles; an entry gets at most 2 contributions from each
    particle of the 2^dims cells around it, each rounded by at most 1/(2S)."""
    t = _brick_shape(dims, nx, ny, nz, capacity)
    nb = [-(-n // t[d]) for d, n in enumerate((nx, ny, nz))]
    i = np.floor(p.x).astype(int) - 3
    j = np.floor(p.y).astype(int) - 3
    k = np.floor(p.z).astype(int) - 3 if dims == 3 else np.zeros_like(i)
    bid = i // t[0] + nb[0] * (j // t[1] + nb[1] * (k // t[2]))
    nmax = max(int(np.bincount(bid).max()), 256)
    per_cell = int(np.bincount(i + nx * (j + ny * k)).max())
    s_min = 2.0 ** 30 / (c * qi * np.abs(p.q).max() * nmax)
    return 2 * (2 ** dims) * per_cell * 0.5 / s_min


@pytest.mark.parametrize("dims", [2, 3])
def test_fp32_tiled_mover_matches_global_mover(dims):
    """The tiled FP32 mover (shared-memory fields, fixed-point current per
    brick) and the per-particle FP32 mover give bit-identical particles and,
    once the ghost current is folded, the same current up to the FP32
    rounding of the summation order plus the bound of the fixed-point
    rounding."""
    nx, ny, nz = (48, 40, 1) if dims == 2 else (24, 16, 12)
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, precision="fp32", qi=0.00158203125, capacity=1 << 18)
    f = random_fields(g, seed=41, scale=0.02)
    with _sim(cfg) as s:
        s.init_weibel(8, 0.5, 0.4, 0.005, 0.005, 9)
        s.reorder()                       # bricks valid -> tiled mover
        sorted_p = s.fetch_particles()
        s.load_fields(to_gpu_fields(f))
        s.move_deposit()
        s.fold_current()
        a_p, a_f = s.fetch_particles(), s.fetch_fields()
        s.load_particles(sorted_p)        # same state, bricks invalid -> per-particle mover
        s.load_fields(to_gpu_fields(f))
        s.move_deposit()
        s.fold_current()
        b_p, b_f = s.fetch_particles(), s.fetch_fields()
    for k in ("x", "y", "z", "u", "v", "w"):
        np.testing.assert_array_equal(getattr(a_p, k), getattr(b_p, k), err_msg=k)
    slack = _fixed_point_slack(sorted_p, dims, nx, ny, nz, 1 << 18, 0.45, 0.00158203125)
    for n in ("Jx", "Jy", "Jz"):
        a, b = interior(getattr(a_f, n), g), interior(getattr(b_f, n), g)
        np.testing.assert_allclose(a, b, rtol=0, atol=2e-6 * np.abs(b).max() + slack, err_msg=n)
        assert slack < 1e-3 * np.abs(b).max()     # the bound itself is small


def _brick_shape(dims, nx, ny, nz, capacity):
    """Brick shape the library picks: about 4096 particles per brick at
    capacity / cells, from a fixed ladder of shapes, clipped to the grid."""
    ladder = [(4, 4, 4), (8, 4, 4), (8, 8, 4), (8, 8, 8)] if dims == 3 else \
        [(8, 8, 1), (16, 8, 1), (16, 16, 1), (32, 16, 1), (32, 32, 1)]
    cells = nx * ny * (nz if dims == 3 else 1)
    target = 4096.0 / max(capacity / cells, 0.5)
    t = next((s for s in ladder if s[0] * s[1] * s[2] >= target), ladder[-1])
    n = (nx, ny, nz)
    return tuple(min(t[d], n[d]) if d < dims else 1 for d in range(3))


def _clumped_particles(dims, nx, ny, nz, clump, seed):
    """Two particles per cell plus `clump` particles packed into one cell
    (its brick then holds more particles than the in-brick order stages in
    shared memory, and the mover's fixed-point scale comes from that count),
    momenta up to 0.4 per component, charges +-1."""
    from pictor_b200 import Particles

    rng = np.random.default_rng(seed)
    cells = nx * ny * (nz if dims == 3 else 1)
    n0 = 2 * cells
    ci = np.repeat(np.arange(cells), 2)
    i, j, k = ci % nx, (ci // nx) % ny, ci // (nx * ny)
    x = 3 + i + rng.uniform(0, 1, n0)
    y = 3 + j + rng.uniform(0, 1, n0)
    z = (3 + k + rng.uniform(0, 1, n0)) if dims == 3 else rng.uniform(1, 2, n0)
    cx, cy, cz = 3 + nx // 3, 3 + ny // 2, 3 + (nz // 2 if dims == 3 else 0)
    x = np.concatenate([x, cx + rng.uniform(0.05, 0.95, clump)])
    y = np.concatenate([y, cy + rng.uniform(0.05, 0.95, clump)])
    z = np.concatenate([z, (cz + rng.uniform(0.05, 0.95, clump)) if dims == 3 else rng.uniform(1, 2, clump)])
    n = n0 + clump
    u, v, w = (rng.uniform(-0.4, 0.4, n) for _ in range(3))
    flv = rng.integers(1, 3, n).astype(np.int32)
    q = np.where(flv == 1, 1.0, -1.0)
    return Particles(q, x, y, z, u, v, w, flv)


@pytest.mark.parametrize("dims", [2, 3])
def test_fp32_dense_brick(dims):
    """A cell holding 12 000 particles: the reorder orders that brick without
    staging (its slots written directly), keeps every particle once, groups
    by brick; the tiled mover, with the scale of that brick, moves the
    particles bit-identically to the per-particle mover and deposits the same
    current up to FP32 summation order and the fixed-point bound."""
    nx, ny, nz = (48, 40, 1) if dims == 2 else (24, 16, 12)
    cap = 1 << 17
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, precision="fp32", qi=0.00158203125, capacity=cap)
    f = random_fields(g, seed=43, scale=0.02)
    p = _clumped_particles(dims, nx, ny, nz, 12000, 17)
    with _sim(cfg) as s:
        s.load_particles(p)
        before = s.fetch_particles()
        s.reorder()
        sorted_p = s.fetch_particles()
        assert s.device_errors() == 0
        s.load_fields(to_gpu_fields(f))
        s.move_deposit()
        s.fold_current()
        a_p, a_f = s.fetch_particles(), s.fetch_fields()
        s.load_particles(sorted_p)        # same state, bricks invalid -> per-particle mover
        s.load_fields(to_gpu_fields(f))
        s.move_deposit()
        s.fold_current()
        b_p, b_f = s.fetch_particles(), s.fetch_fields()
    assert len(sorted_p.x) == len(p.x)
    t = _brick_shape(dims, nx, ny, nz, cap)
    nb = [-(-n // t[d]) for d, n in enumerate((nx, ny, nz))]
    i = np.floor(sorted_p.x).astype(int) - 3
    j = np.floor(sorted_p.y).astype(int) - 3
    k = np.floor(sorted_p.z).astype(int) - 3 if dims == 3 else np.zeros_like(i)
    bid = i // t[0] + nb[0] * (j // t[1] + nb[1] * (k // t[2]))
    assert np.all(np.diff(bid) >= 0) and np.bincount(bid).max() > 8192
    key = lambda q: np.lexsort((q.w, q.v, q.u, q.z, q.y, q.x))
    ka, kb = key(sorted_p), key(before)
    for fld in ("x", "y", "z", "u", "v", "w", "q", "flv"):
        np.testing.assert_array_equal(getattr(sorted_p, fld)[ka], getattr(before, fld)[kb], err_msg=fld)
    for fld in ("x", "y", "z", "u", "v", "w"):
        np.testing.assert_array_equal(getattr(a_p, fld), getattr(b_p, fld), err_msg=fld)
    # the worst-case fixed-point bound grows with the 12 000 contributions of
    # the packed cell (whose +-1 charges with random momenta mostly cancel),
    # so the observed difference is held to 1e-4 of the largest entry as well
    slack = _fixed_point_slack(sorted_p, dims, nx, ny, nz, cap, 0.45, 0.00158203125)
    for n in ("Jx", "Jy", "Jz"):
        a, b = interior(getattr(a_f, n), g), interior(getattr(b_f, n), g)
        np.testing.assert_allclose(a, b, rtol=0, atol=2e-6 * np.abs(b).max() + slack, err_msg=n)
        assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max(), n


@pytest.mark.parametrize("dims", [2, 3])
def test_fp32_reorder_groups_by_brick(dims):
    """The FP32 reorder keeps every live particle once, drops holes, and
    groups the particles by brick in increasing brick order."""
    nx, ny, nz = (40, 36, 1) if dims == 2 else (20, 16, 12)
    cap = 1 << 16
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, precision="fp32", qi=0.00158203125, capacity=cap)
    with _sim(cfg) as s:
        n0 = s.init_weibel(8, 0.5, 0.4, 0.005, 0.005, 5)
        before = s.fetch_particles()
        s.reorder()
        after = s.fetch_particles()
    assert len(after.x) == n0 and np.all(after.flv > 0)
    t = _brick_shape(dims, nx, ny, nz, cap)
    nb = [-(-n // t[d]) for d, n in enumerate((nx, ny, nz))]
    i = np.floor(after.x).astype(int) - 3
    j = np.floor(after.y).astype(int) - 3
    k = np.floor(after.z).astype(int) - 3 if dims == 3 else np.zeros_like(i)
    bid = i // t[0] + nb[0] * (j // t[1] + nb[1] * (k // t[2]))
    assert np.all(np.diff(bid) >= 0)
    key = lambda p: np.lexsort((p.w, p.v, p.u, p.z, p.y, p.x))
    ka, kb = key(after), key(before)
    for f in ("x", "y", "z", "u", "v", "w", "q", "flv"):
        np.testing.assert_array_equal(getattr(after, f)[ka], getattr(before, f)[kb], err_msg=f)


@pytest.mark.parametrize("dims", [2, 3])
def test_fp32_tiled_steps_track_per_particle_steps(dims):
    """40 steps without a reorder after the first one: the bricks' particles
    drift well past their bricks (boxes grow, some fall back to the brick plus
    one cell with the rest of the particles through global memory, some cross
    the periodic boundary) and the run stays on the per-particle run up to
    FP32 summation-order noise."""
    nx, ny, nz = (48, 40, 1) if dims == 2 else (24, 16, 16)
    res = {}
    for tiled in (True, False):
        g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, precision="fp32", qi=0.00158203125,
                                 capacity=1 << 18, reorder_period=0)
        with _sim(cfg) as s:
            s.init_weibel(8, 0.5, 0.8, 0.01, 0.01, 77)
            if tiled:
                s.reorder()
            s.step(40)
            res[tiled] = s.diagnostics(0.00158203125)
    a, b = res[True], res[False]
    np.testing.assert_allclose(a["kinetic"], b["kinetic"], rtol=1e-5)
    assert abs((a["B2"] + a["E2"]) - (b["B2"] + b["E2"])) <= 1e-3 * (b["B2"] + b["E2"])


@pytest.mark.parametrize("dims", [2, 3])
def test_fp32_form_tracks_fp64(dims):
    """FP32 cell-relative run vs the FP64 reference form from the same seed:
    energies agree to the stated tolerance after 30 steps."""
    nx, ny, nz = (64, 64, 1) if dims == 2 else (24, 24, 24)
    res = {}
    for prec in ("fp64", "fp32"):
        g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, precision=prec, qi=0.00158203125, capacity=1 << 19)
        with _sim(cfg) as s:
            s.init_weibel(16 if dims == 2 else 4, 0.5, 0.5, 0.005, 0.005, 2930)
            s.reorder()
            s.step(30)
            d = s.diagnostics(0.00158203125)
            res[prec] = d
    a, b = res["fp32"], res["fp64"]
    tot32 = 0.5 * (a["B2"] + a["E2"]) + a["kinetic"].sum()
    tot64 = 0.5 * (b["B2"] + b["E2"]) + b["kinetic"].sum()
    assert abs(tot32 - tot64) <= 1e-5 * abs(tot64)
    fe32, fe64 = a["B2"] + a["E2"], b["B2"] + b["E2"]
    assert abs(fe32 - fe64) <= 1e-2 * fe64
    # both forms keep the reference's weights, which conserve charge exactly
    # in 2D and not in 3D
    assert a["gauss_linf"] <= (1e-4 if dims == 2 else 2e-2) * a["rho_max"]
    assert b["gauss_linf"] <= (1e-12 if dims == 2 else 1e-2) * b["rho_max"]


def test_fp32_exact_charge_conserves_charge():
    """The FP32 3D form with pic_config.exact_charge: each zigzag segment
    deposits its exact line integral (cross term q dx dy dz / 12), so the
    Gauss residual stays at FP32 round-off (1e-4 of the peak charge density
    over 60 steps, against 2e-2 with the reference's weights), by tiles and
    per particle alike, and the energies follow the FP64 form's."""
    nx, ny, nz = 24, 24, 24
    res = {}
    for tiled in (True, False):
        g, cfg = grid_and_config(dims=3, nx=nx, ny=ny, nz=nz, precision="fp32", qi=0.00158203125,
                                 capacity=1 << 19, reorder_period=20 if tiled else 0)
        cfg.exact_charge = 1
        with _sim(cfg) as s:
            s.init_weibel(4, 0.5, 0.5, 0.005, 0.005, 2930)
            if tiled:
                s.reorder()
            s.step(60)
            res[tiled] = s.diagnostics(0.00158203125)
    for d in res.values():
        assert d["gauss_linf"] <= 1e-4 * d["rho_max"], d
    a, b = res[True], res[False]
    np.testing.assert_allclose(a["kinetic"], b["kinetic"], rtol=1e-5)


# ---------------------------------------------------------------------------
# Cylindrical (r, theta, z) FP64 form vs the cylindrical restatement
# ---------------------------------------------------------------------------
def _cyl(fdtd="yee", nx=12, ny=8, nz=10, capacity=1 << 15, reorder_period=20):
    from pictor_b200 import PicConfig

    g = O.make_grid(3, nx, ny, nz, c=0.45, qi=0.01, fdtd=fdtd, qm=(1.0, -1.0))
    cfg = PicConfig(nx=nx, ny=ny, nz=nz, dims=3, c=0.45, qi=0.01, qm=(1.0, -1.0), fdtd=fdtd, geom="cylindrical",
                    capacity=capacity, reorder_period=reorder_period, rmin=-0.5, inc_axis=1)
    return g, cfg


def _cyl_particles(g, seed=3):
    p = O.cyl_load_uniform(g, 1, 1, 1, 1.0, 2e-3, -1.0, 2, seed, 1 << 14)
    rng = np.random.default_rng(seed)
    n = p.used
    # a few near-axis particles moving through the axis region, and some ions
    k = min(40, n)
    idx = rng.choice(n, k, replace=False)
    p.x[idx] = 3.5 + rng.uniform(0.05, 1.0, k)
    p.u[idx] = rng.uniform(-0.6, 0.6, k)
    p.v[idx] = rng.uniform(-0.6, 0.6, k)
    p.flv[idx[: k // 2]] = 1
    p.q[idx[: k // 2]] *= -1.0
    return p


@pytest.mark.parametrize("fdtd", ["yee", "lehe"])
def test_cyl_field_phases_bit_exact(fdtd):
    g, cfg = _cyl(fdtd)
    f = random_fields(g, seed=51, consistent_ghosts=False)
    o = O.CylOracle(g, O.Particles(1), f.copy())
    with _sim(cfg) as s:
        s.load_fields(to_gpu_fields(f))
        o.update_b_half(); o.send_recv_flds("B")
        s.update_b_half()
        gf = s.fetch_fields()
        for n in ("Bx", "By", "Bz"):
            assert np.array_equal(getattr(gf, n), getattr(o.f, n)), n
        o.update_e(); o.send_recv_flds("E")
        s.update_e()
        gf = s.fetch_fields()
        for n in ("Ex", "Ey", "Ez"):
            assert np.array_equal(getattr(gf, n), getattr(o.f, n)), n
        rng = np.random.default_rng(6)
        J = [np.asfortranarray(rng.normal(scale=1e-3, size=O.grid_shape(g))) for _ in range(3)]
        o.f.Jx[...], o.f.Jy[...], o.f.Jz[...] = J
        s.load_current(*J)
        o.fold_current(); s.fold_current()
        gf = s.fetch_fields()
        for n in ("Jx", "Jy", "Jz"):
            assert np.array_equal(getattr(gf, n), getattr(o.f, n)), n
        o.add_current(); o.send_recv_flds("E")
        s.add_current()
        gf = s.fetch_fields()
        for n in ("Ex", "Ey", "Ez"):
            assert np.array_equal(getattr(gf, n), getattr(o.f, n)), n


def test_cyl_move_deposit_and_exchange_parity():
    g, cfg = _cyl()
    f = random_fields(g, seed=52, scale=0.02, consistent_ghosts=False)
    p = _cyl_particles(g)
    o = O.CylOracle(g, p.copy(), f.copy())
    with _sim(cfg) as s:
        s.load_fields(to_gpu_fields(f))
        s.load_particles(to_gpu_particles(p))
        o.move_deposit(); s.move_deposit()
        # the azimuthal move calls atan (device vs libm: last-ulp differences), so
        # positions agree to round-off; momenta and cells match
        gp = s.fetch_particles()
        assert_particles_equal(gp, o.p, exact=False, rtol=1e-13)
        v = o.p.view()
        for k in ("x", "y", "z"):
            assert np.array_equal(np.floor(getattr(gp, k)), np.floor(v[k])), k
        gf = s.fetch_fields()
        for n in ("Jx", "Jy", "Jz"):
            a, b = getattr(gf, n), getattr(o.f, n)
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * np.abs(b).max(), err_msg=n)
        assert o.exchange_particles() == 0
        s.exchange_particles()
        assert s.particle_count() == o.p.used
        assert_particles_equal(s.fetch_particles(), o.p, exact=False, rtol=1e-13)


def test_cyl_tiled_f64_mover_after_reorder():
    """After a reorder the FP64 cylindrical mover runs by tiles (the staged
    node box serves both gathers of the Strang split, a 64-bit fixed-point
    current box): three moves with exchanges in between against the oracle
    (positions to round-off, the device atan; cells exact; J to 1e-12 of its
    scale), and the same moves per particle (fp64_tiles = -1) give the
    tiled form's positions and momenta bit for bit."""
    g, cfg = _cyl(nx=16, ny=12, nz=12, capacity=1 << 16)
    f = random_fields(g, seed=53, scale=0.02, consistent_ghosts=False)
    p = _cyl_particles(g, seed=8)
    o = O.CylOracle(g, p.copy(), f.copy())
    got = {}
    for tiles in (1, -1):
        cfg.fp64_tiles = tiles
        with _sim(cfg) as s:
            s.load_fields(to_gpu_fields(f))
            s.load_particles(to_gpu_particles(p))
            s.reorder()
            if tiles == 1:
                o.reorder()
            snaps = []
            for it in range(3):
                s.move_deposit()
                snaps.append(s.fetch_particles())
                if tiles == 1:
                    o.move_deposit()
                    gp = snaps[-1]
                    assert_particles_equal(gp, o.p, exact=False, rtol=1e-13)
                    v = o.p.view()
                    for k in ("x", "y", "z"):
                        assert np.array_equal(np.floor(getattr(gp, k)), np.floor(v[k])), k
                    gf = s.fetch_fields()
                    for n in ("Jx", "Jy", "Jz"):
                        a, b = getattr(gf, n), getattr(o.f, n)
                        np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * np.abs(b).max(), err_msg=n)
                    assert o.exchange_particles() == 0
                s.exchange_particles()
            assert s.device_errors() == 0
            got[tiles] = snaps
    for a, b in zip(got[1], got[-1]):
        for k in ("q", "x", "y", "z", "u", "v", "w", "flv"):
            assert np.array_equal(getattr(a, k), getattr(b, k)), k


@pytest.mark.parametrize("fdtd", ["yee", "lehe"])
def test_cyl_full_steps_lockstep(fdtd):
    g, cfg = _cyl(fdtd, reorder_period=4)
    p = _cyl_particles(g, seed=4)
    o = O.CylOracle(g, p.copy())
    with _sim(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        o.step(1, 4); s.step(1)
        assert_particles_equal(s.fetch_particles(), o.p, exact=False, rtol=1e-13)
        for t in range(2, 9):
            o.step(t, 4); s.step(1)
        assert s.particle_count() == o.p.used
        gp, v = s.fetch_particles(), o.p.view()
        assert np.array_equal(gp.flv, v["flv"])
        for k in ("x", "y", "z", "u", "v", "w"):
            np.testing.assert_allclose(getattr(gp, k), v[k], rtol=1e-9, atol=1e-9, err_msg=k)
        gf = s.fetch_fields(with_current=False)
        for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
            a, b = getattr(gf, n), getattr(o.f, n)
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-9 * max(np.abs(b).max(), 1e-30), err_msg=n)


def test_cyl_wakefield_lockstep():
    """A relativistic (gamma 50) electron bunch crossing the axis of an
    r-weighted plasma, Lehe along z, Courant 0.3: 6 steps of the CUDA path
    against the oracle's cylindrical step."""
    from pictor_b200 import PicConfig, init_scale
    from pictor_b200.setups import cyl_wakefield

    nr, nt, nz, c = 20, 8, 48, 0.3
    qi = init_scale(c, 10.0, 8)["qi"]
    gp, _ = cyl_wakefield(nr, nz, nt, c, bunch_sigma_r=3.0, bunch_sigma_z=5.0, bunch_particles=4096, seed=11)
    n = len(gp.x)
    g = O.make_grid(3, nr, nt, nz, c=c, qi=qi, fdtd="lehe", qm=(1.0, -1.0))
    cfg = PicConfig(nx=nr, ny=nt, nz=nz, dims=3, c=c, qi=qi, qm=(1.0, -1.0), fdtd="lehe", geom="cylindrical",
                    capacity=3 * n, reorder_period=4, rmin=-0.5, inc_axis=1)
    o = O.CylOracle(g, O.Particles.from_arrays(3 * n, **{k: getattr(gp, k) for k in gp.NAMES}))
    with _sim(cfg) as s:
        s.load_particles(gp)
        for t in range(1, 7):
            o.step(t, 4)
            s.step(1)
        assert s.particle_count() == o.p.used
        sp, v = s.fetch_particles(), o.p.view()
        assert np.array_equal(sp.flv, v["flv"])
        for k in ("x", "y", "z", "u", "v", "w"):
            np.testing.assert_allclose(getattr(sp, k), v[k], rtol=1e-9, atol=1e-9, err_msg=k)
        gf = s.fetch_fields(with_current=False)
        for name in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
            a, b = getattr(gf, name), getattr(o.f, name)
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-9 * max(np.abs(b).max(), 1e-30), err_msg=name)
        assert np.abs(gf.Ez).max() > 0


@pytest.mark.parametrize("fdtd", ["yee", "lehe"])
def test_cyl_fp32_field_phases_track_fp64(fdtd):
    """The FP32 cylindrical form's field phases (B half step with the axis
    updates, E update, fold, AddCurrent) equal the FP64 ones to FP32
    rounding (1e-6 of the field scale)."""
    g, cfg64 = _cyl(fdtd)
    _, cfg32 = _cyl(fdtd)
    cfg32.precision = "fp32"
    f = random_fields(g, seed=51, consistent_ghosts=False)
    rng = np.random.default_rng(6)
    J = [np.asfortranarray(rng.normal(scale=1e-3, size=O.grid_shape(g))) for _ in range(3)]
    out = {}
    for name, cfg in (("fp64", cfg64), ("fp32", cfg32)):
        with _sim(cfg) as s:
            s.load_fields(to_gpu_fields(f))
            s.update_b_half()
            s.update_e()
            s.load_current(*J)
            s.fold_current()
            s.add_current()
            out[name] = s.fetch_fields()
    for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Jx", "Jy", "Jz"):
        a, b = getattr(out["fp32"], n), getattr(out["fp64"], n)
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-6 * np.abs(b).max(), err_msg=n)


def test_cyl_fp32_mover_tracks_fp64():
    """One push + deposit of the FP32 cell-relative cylindrical mover against
    the FP64 one on the same particles (including near-axis particles, which
    take the sub-stepper) and fields: positions to 1e-5 of a cell (the FP64
    ones wrapped in theta and z as the FP32 mover does), momenta to 1e-5
    relative, and the folded current to 1e-4 of its scale."""
    g, cfg64 = _cyl("lehe", capacity=1 << 15)
    _, cfg32 = _cyl("lehe", capacity=1 << 15)
    cfg32.precision = "fp32"
    f = random_fields(g, seed=57, scale=0.02)
    p = _cyl_particles(g, seed=8)
    # keep clear of the outer radius (the FP32 mover drops leavers at once)
    keep = p.x[:p.used] < g.mx - 4.0
    n = int(keep.sum())
    gp = to_gpu_particles(p)
    from pictor_b200 import Particles

    gp = Particles(*(getattr(gp, k)[:p.used][keep].copy() for k in gp.NAMES))
    out = {}
    for name, cfg in (("fp64", cfg64), ("fp32", cfg32)):
        with _sim(cfg) as s:
            s.load_particles(gp)
            s.load_fields(to_gpu_fields(f))
            s.move_deposit()
            s.fold_current()
            assert s.device_errors() == 0
            out[name] = (s.fetch_particles(), s.fetch_fields())
    (p64, f64), (p32, f32) = out["fp64"], out["fp32"]
    assert len(p32.x) == len(p64.x) == n
    ylo, ylen = 3.0, g.my - 5.0
    zlo, zlen = 3.0, g.mz - 5.0
    y64 = (p64.y - ylo) % ylen + ylo
    z64 = (p64.z - zlo) % zlen + zlo
    np.testing.assert_allclose(p32.x, p64.x, rtol=0, atol=1e-5)
    dy = np.abs(p32.y - y64)
    assert np.minimum(dy, ylen - dy).max() < 1e-5
    dz = np.abs(p32.z - z64)
    assert np.minimum(dz, zlen - dz).max() < 1e-5
    for k in ("u", "v", "w"):
        a, b = getattr(p32, k), getattr(p64, k)
        np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-6 * np.abs(b).max(), err_msg=k)
    for nme in ("Jx", "Jy", "Jz"):
        a, b = interior(getattr(f32, nme), g), interior(getattr(f64, nme), g)
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-4 * np.abs(b).max(), err_msg=nme)


def test_cyl_fp32_steps_track_fp64():
    """The wakefield case of test_cyl_wakefield_lockstep, 20 steps in the
    FP32 form against the FP64 form: particle count equal, field energy
    within 1e-3 and kinetic energy within 1e-5."""
    from pictor_b200 import PicConfig, Simulation, init_scale
    from pictor_b200.setups import cyl_wakefield

    nr, nt, nz, c = 20, 8, 48, 0.3
    qi = init_scale(c, 10.0, 8)["qi"]
    gp, _ = cyl_wakefield(nr, nz, nt, c, bunch_sigma_r=3.0, bunch_sigma_z=5.0, bunch_particles=4096, seed=11)
    res = {}
    for prec in ("fp64", "fp32"):
        cfg = PicConfig(nx=nr, ny=nt, nz=nz, dims=3, c=c, qi=qi, qm=(1.0, -1.0), fdtd="lehe", geom="cylindrical",
                        precision=prec, capacity=3 * len(gp.x), reorder_period=10, rmin=-0.5, inc_axis=1)
        with Simulation(cfg) as s:
            s.load_particles(gp)
            s.step(20)
            assert s.device_errors() == 0
            res[prec] = (s.particle_count(), s.diagnostics())
    (n64, d64), (n32, d32) = res["fp64"], res["fp32"]
    assert n32 == n64
    fe64, fe32 = d64["B2"] + d64["E2"], d32["B2"] + d32["E2"]
    assert abs(fe32 - fe64) <= 1e-3 * fe64
    np.testing.assert_allclose(d32["kinetic"].sum(), d64["kinetic"].sum(), rtol=1e-5)


def test_cyl_field_energy_matches_oracle():
    g, cfg = _cyl()
    f = random_fields(g, seed=53, consistent_ghosts=False)
    o = O.CylOracle(g, O.Particles(1), f.copy())
    with _sim(cfg) as s:
        s.load_fields(to_gpu_fields(f))
        d = s.diagnostics()
    eb, ee = o.field_energy()
    np.testing.assert_allclose([d["B2"], d["E2"]], [eb, ee], rtol=1e-12)
