"""The tiled FP32 cylindrical mover (one CTA per brick, node-averaged fields
and a 64-bit fixed-point current box in shared memory, the radius not
periodic) against the per-particle FP32 cylindrical mover: particles bit for
bit, currents up to FP32 rounding and summation order."""
import numpy as np
import pytest

from oracle import oracle as O

from ._util import interior, random_fields, to_gpu_fields
from .test_gpu_parity import _brick_shape

pytestmark = pytest.mark.gpu

QI = 0.01


def _cfg(nx, ny, nz, capacity, fdtd="lehe", reorder_period=0):
    from pictor_b200 import PicConfig

    g = O.make_grid(3, nx, ny, nz, c=0.45, qi=QI, fdtd=fdtd, qm=(1.0, -1.0))
    cfg = PicConfig(nx=nx, ny=ny, nz=nz, dims=3, c=0.45, qi=QI, qm=(1.0, -1.0), fdtd=fdtd, geom="cylindrical",
                    precision="fp32", capacity=capacity, reorder_period=reorder_period, rmin=-0.5, inc_axis=1)
    return g, cfg


def _particles(g, n, seed):
    """Particles over the whole cylinder: a fifth near the axis (x < 4.5, the
    sub-stepper), some just inside the outer radius moving out (they leave),
    some on the theta and z seams; momenta up to 0.5 per component."""
    from pictor_b200 import Particles

    rng = np.random.default_rng(seed)
    x = rng.uniform(3.5, g.mx - 2.0, n)
    near = rng.random(n) < 0.2
    x[near] = rng.uniform(3.5, 4.5, near.sum())
    y = rng.uniform(3.0, g.my - 2.0, n)
    z = rng.uniform(3.0, g.mz - 2.0, n)
    seam = rng.random(n) < 0.1
    y[seam] = rng.choice([3.02, g.my - 2.02], seam.sum())
    z[~seam & (rng.random(n) < 0.1)] = g.mz - 2.05
    u, v, w = (rng.uniform(-0.5, 0.5, n) for _ in range(3))
    out = x > g.mx - 3.3
    u[out] = np.abs(u[out]) + 0.2
    flv = rng.integers(1, 3, n).astype(np.int32)
    q = np.where(flv == 1, 1.0, -1.0) * (x - 3.0)     # weights by r, as the cylindrical loader sets them
    return Particles(q, x, y, z, u, v, w, flv)


def _brick_max(p, t, nx, ny, nz):
    i = np.floor(p.x).astype(int) - 3
    j = np.floor(p.y).astype(int) - 3
    k = np.floor(p.z).astype(int) - 3
    nb = [-(-a // b) for a, b in zip((nx, ny, nz), t)]
    bid = i // t[0] + nb[0] * (j // t[1] + nb[1] * (k // t[2]))
    return max(int(np.bincount(bid).max()), 256), int(np.bincount(i + nx * (j + ny * k)).max())


def test_cyl_tiled_mover_matches_per_particle_mover():
    """One push + deposit after a reorder (tiled) and of the same particles
    reloaded (per-particle): every position and momentum equal, the same
    particles dropped at the outer radius, and the folded current equal up to
    FP32 rounding and summation order: the box adds each contribution as an
    FP32 value scaled by S = 2^62 / (2 qi max|w| max(N, 256)) and rounded to
    a 64-bit integer, so the integer rounding (the slack below) is far
    below the FP32 rounding of the contribution itself, weights near the
    axis 20 times below the largest included."""
    from pictor_b200 import Simulation

    nx, ny, nz = 24, 8, 16
    g, cfg = _cfg(nx, ny, nz, capacity=1 << 16)
    f = random_fields(g, seed=61, scale=0.02)
    gp = _particles(g, 12000, seed=5)
    with Simulation(cfg) as s:
        s.load_particles(gp)
        s.reorder()                        # bricks valid -> tiled mover
        sorted_p = s.fetch_particles()
        s.load_fields(to_gpu_fields(f))
        s.move_deposit()
        s.fold_current()
        assert s.device_errors() == 0
        a_p, a_f = s.fetch_particles(), s.fetch_fields()
        s.load_particles(sorted_p)         # same order, bricks invalid -> per-particle mover
        s.load_fields(to_gpu_fields(f))
        s.move_deposit()
        s.fold_current()
        assert s.device_errors() == 0
        b_p, b_f = s.fetch_particles(), s.fetch_fields()
    live = [int((q.flv != 0).sum()) for q in (a_p, b_p, sorted_p)]
    assert live[0] == live[1] < live[2]     # the same particles left through the outer radius
    for k in ("x", "y", "z", "u", "v", "w", "q", "flv"):
        np.testing.assert_array_equal(getattr(a_p, k), getattr(b_p, k), err_msg=k)
    nmax, per_cell = _brick_max(sorted_p, _brick_shape(3, nx, ny, nz, 1 << 16), nx, ny, nz)
    s_min = 2.0 ** 62 / (2.0 * QI * np.abs(sorted_p.q).max() * nmax)
    slack = 8 * per_cell * 0.5 / s_min
    for n in ("Jx", "Jy", "Jz"):
        a, b = interior(getattr(a_f, n), g), interior(getattr(b_f, n), g)
        np.testing.assert_allclose(a, b, rtol=0, atol=2e-6 * np.abs(b).max() + slack, err_msg=n)
        assert slack < 1e-10 * np.abs(b).max()     # the bound itself is negligible


@pytest.mark.parametrize("modes", [0, 2])
def test_cyl_tiled_steps_track_per_particle_steps(modes):
    """The wakefield case (weights by radius, a cold background whose
    currents are small next to the bunch's), 30 steps without a reorder
    after the first one (the bunch drifts 9 cells in z, past its bricks'
    boxes), theta-gridded and modal field solves: the tiled run stays on the
    per-particle run up to FP32 summation-order noise (same particle count,
    kinetic energy 1e-6, field energy 1e-5)."""
    from pictor_b200 import PicConfig, Simulation, init_scale
    from pictor_b200.setups import cyl_wakefield

    nr, nt, nz, c = 20, 8, 48, 0.3
    qi = init_scale(c, 10.0, 8)["qi"]
    gp, _ = cyl_wakefield(nr, nz, nt, c, bunch_sigma_r=3.0, bunch_sigma_z=5.0, bunch_particles=4096, seed=13)
    res = {}
    for tiled in (True, False):
        cfg = PicConfig(nx=nr, ny=nt, nz=nz, dims=3, c=c, qi=qi, qm=(1.0, -1.0), fdtd="lehe", geom="cylindrical",
                        precision="fp32", capacity=3 * len(gp.x), reorder_period=0, rmin=-0.5, inc_axis=1,
                        cyl_modes=modes)
        with Simulation(cfg) as s:
            s.load_particles(gp)
            if tiled:
                s.reorder()
            s.step(30)
            assert s.device_errors() == 0
            res[tiled] = (s.particle_count(), s.diagnostics())
    (na, da), (nb, db) = res[True], res[False]
    assert na == nb
    np.testing.assert_allclose(da["kinetic"].sum(), db["kinetic"].sum(), rtol=1e-6)
    fa, fb = da["B2"] + da["E2"], db["B2"] + db["E2"]
    assert abs(fa - fb) <= 1e-5 * fb, (fa, fb)
