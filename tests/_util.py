"""Shared fixtures for the parity tests: seeded random states that the oracle
and the CUDA path start from, and the comparisons between them."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O


def grid_and_config(dims=2, nx=16, ny=12, nz=10, fdtd="yee", precision="fp64", c=0.45, qi=0.0123,
                    qm=(1.0, -1.0), bext=(0.0, 0.0, 0.0), capacity=1 << 16, reorder_period=20, curr_filter=0):
    from pictor_b200 import PicConfig

    g = O.make_grid(dims, nx, ny, nz, c=c, qi=qi, fdtd=fdtd, qm=qm, bext=bext)
    cfg = PicConfig(nx=nx, ny=ny, nz=nz, dims=dims, c=c, qi=qi, qm=qm, fdtd=fdtd, precision=precision, bext=bext,
                    capacity=capacity, reorder_period=reorder_period, curr_filter=curr_filter)
    return g, cfg


def random_fields(g, seed=1, scale=0.05, consistent_ghosts=True) -> O.Fields:
    """Random E and B; ghosts made periodic images with the oracle halo."""
    rng = np.random.default_rng(seed)
    f = O.Fields(g)
    for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        getattr(f, n)[...] = rng.normal(scale=scale, size=O.grid_shape(g))
    if consistent_ghosts:
        o = O.Oracle(g, O.Particles(1), f)
        o.send_recv_flds("E")
        o.send_recv_flds("B")
    return f


def random_particles(g, n=4000, seed=2, umax=0.8, holes=0.05, near_boundary=0.2, capacity=None) -> O.Particles:
    """Particles in the interior [3, m-2) with a fraction close to the faces
    (so that they leave through the periodic boundaries) and some holes."""
    rng = np.random.default_rng(seed)
    cap = capacity or (3 * n + 64)
    p = O.Particles(cap)
    x = rng.uniform(3.0, g.mx - 2.0, n)
    y = rng.uniform(3.0, g.my - 2.0, n)
    nb = rng.random(n) < near_boundary
    side = rng.random(n) < 0.5
    x[nb & side] = rng.choice([3.0, g.mx - 2.0], size=(nb & side).sum()) + rng.uniform(-0.0, 0.4, (nb & side).sum()) * np.where(rng.random((nb & side).sum()) < 0.5, 1, -1)
    y[nb & ~side] = rng.choice([3.0, g.my - 2.0], size=(nb & ~side).sum()) + rng.uniform(-0.0, 0.4, (nb & ~side).sum()) * np.where(rng.random((nb & ~side).sum()) < 0.5, 1, -1)
    x = np.clip(x, 3.0, g.mx - 2.0 - 1e-9)
    y = np.clip(y, 3.0, g.my - 2.0 - 1e-9)
    if g.dims == 3:
        z = rng.uniform(3.0, g.mz - 2.0, n)
        nbz = rng.random(n) < near_boundary / 2
        z[nbz] = rng.choice([3.0, g.mz - 2.0 - 1e-9], size=nbz.sum())
        z = np.clip(z, 3.0, g.mz - 2.0 - 1e-9)
    else:
        z = rng.uniform(1.0, 2.0, n)
    u = rng.uniform(-umax, umax, (3, n))
    flv = rng.integers(1, 3, n).astype(np.int32)
    q = np.where(flv == 1, 1.0, -1.0) * rng.uniform(0.5, 1.5, n)
    hole = rng.random(n) < holes
    flv[hole] = 0
    q[hole] = 0.0
    u[:, hole] = 0.0
    x[hole] = 3.8
    y[hole] = 3.8
    z[hole] = 3.8 if g.dims == 3 else 1.5
    for k, a in zip(("q", "x", "y", "z", "u", "v", "w", "flv"), (q, x, y, z, u[0], u[1], u[2], flv)):
        getattr(p, k)[:n] = a
    p.used = n
    return p


def to_gpu_particles(p: O.Particles):
    from pictor_b200 import Particles

    v = p.view()
    return Particles(*(v[k].copy() for k in ("q", "x", "y", "z", "u", "v", "w")), v["flv"].astype(np.int32).copy())


def to_gpu_fields(f: O.Fields):
    from pictor_b200 import Fields

    return Fields(*(getattr(f, n).copy(order="F") for n in O.Fields.NAMES))


def interior(a: np.ndarray, g) -> np.ndarray:
    if g.dims == 3:
        return a[2:g.mx - 3, 2:g.my - 3, 2:g.mz - 3]
    return a[2:g.mx - 3, 2:g.my - 3, :]


def assert_particles_equal(gp, op: O.Particles, exact=True, rtol=0.0):
    v = op.view()
    assert len(gp.x) == op.used
    for k in ("q", "x", "y", "z", "u", "v", "w"):
        a, b = getattr(gp, k), v[k]
        if exact:
            bad = np.nonzero(a != b)[0]
            assert bad.size == 0, f"{k}: {bad.size} mismatches, first {bad[:5]}: gpu {a[bad[:5]]} oracle {b[bad[:5]]}"
        else:
            np.testing.assert_allclose(a, b, rtol=rtol, atol=rtol, err_msg=k)
    assert np.array_equal(gp.flv, v["flv"]), "flv mismatch"
