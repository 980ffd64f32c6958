"""The oracle's convolutional PML (src/bc/bc_pml.F90) against a second,
vectorised restatement written here from the same routines: the
coefficients a, b (pml_ab) and c (pml_c) per position with Python's libm
exp, then UpdateElcFld_PML / UpdateMagFld_PML over the 2..m-1 box in numpy
with the reference's operation order; the two must agree bit for bit on
random fields, two calls in a row (the psi grids carry over).  Then the
behaviour the layer exists for: a plane pulse leaving the box through PML
faces loses its energy, where the periodic box keeps it."""
import math

import numpy as np
import pytest

from oracle import oracle as O

HUGE = 2147483647.0
ALPHA = float(np.float32(9.0e-4))   # the default-kind literal of SetPMLParameters


def _profile(faces: dict):
    """pml_pos, pml_pos_ind, L, sigma_max, alpha_max per face 0..5."""
    pos, ind, L, smax, amax = [], [], [], [], []
    for f in range(6):
        up = f % 2 == 1
        if f + 1 in faces:
            p, t = faces[f + 1]
            pos.append(p)
            ind.append(math.ceil(p) + 1.0 if up else math.floor(p) - 1.0)
            L.append(t)
            smax.append(1.0)
            amax.append(ALPHA)
        else:
            pos.append(HUGE if up else -HUGE)
            ind.append(HUGE if up else -HUGE)
            L.append(10.0)
            smax.append(0.0)
            amax.append(1.0)
    return pos, ind, L, smax, amax


def _coef(prof, fc, x, axis):
    """(a, b, c) of pml_ab / pml_c; kappa_max = 1 makes kappa 1."""
    pos, _, L, smax, amax = prof
    a = b = c = 0.0
    for f, d in ((2 * axis + 1, x - pos[2 * axis + 1]), (2 * axis, pos[2 * axis] - x)):
        if d > 0:
            t = d / L[f]
            t2 = t * t
            sigma = min(smax[f], smax[f] * (t2 * t2))
            kappa = min(1.0, 1.0 + (t2 * t2) * (1.0 - 1.0))
            alpha = amax[f]
            a = math.exp(-(sigma / kappa) - alpha)
            b = (sigma / (sigma * kappa + alpha * (kappa * kappa))) * (a - 1.0)
            c = fc * (1.0 / kappa - 1.0)
    return a, b, c


def _tables(prof, fc, m, axis, half):
    off = 0.5 if half else 0.0
    rows = [_coef(prof, fc, (a - 3) + off, axis) for a in range(1, m + 1)]
    return [np.array([r[q] for r in rows]) for q in range(3)]


def _beyond(prof, x, axis):
    pos, _, L, _, _ = prof
    return (x < pos[2 * axis] - L[2 * axis]) | (x > pos[2 * axis + 1] + L[2 * axis + 1])


def _restated(g, F, psi, faces, which):
    """UpdateElcFld_PML (which 'E') or UpdateMagFld_PML ('B') over numpy
    copies: F maps component names to (mx, my, mz) arrays, psi the six psi
    grids of that field."""
    prof = _profile(faces)
    d3 = g.dims == 3
    m = (g.mx, g.my, g.mz)
    half = which == "B"
    T = [_tables(prof, g.c, m[a], a, half) for a in range(3)]
    ix = np.arange(2, g.mx)                          # 1-based i = 2..mx-1
    jy = np.arange(2, g.my)
    kz = np.arange(2, g.mz) if d3 else np.array([1])
    I, J, K = np.meshgrid(ix, jy, kz, indexing="ij")
    ind = prof[1]
    inside = ((I - 3 > ind[0]) & (I - 3 < ind[1]) & (J - 3 > ind[2]) & (J - 3 < ind[3]) &
              (K - 3 > ind[4]) & (K - 3 < ind[5]))
    sel = ~inside
    i, j, k = I[sel] - 1, J[sel] - 1, K[sel] - 1     # 0-based
    ax, bx, cx = (t[i] for t in T[0])
    ay, by, cy = (t[j] for t in T[1])
    az, bz, cz = (t[k] for t in T[2])
    fc = g.c
    p1x, p1y, p1z, p2x, p2y, p2z = psi
    s = 1 if which == "B" else -1                    # forward differences for B, backward for E
    src = ("E" if which == "B" else "B")
    Sx, Sy, Sz = F[src + "x"], F[src + "y"], F[src + "z"]

    def dd(A, axis):
        o = [i, j, k]
        o[axis] = o[axis] + s
        return (A[tuple(o)] - A[i, j, k]) if s == 1 else (A[i, j, k] - A[tuple(o)])

    p1x[i, j, k] = ay * p1x[i, j, k] + (by * fc) * dd(Sz, 1)
    p1z[i, j, k] = ax * p1z[i, j, k] + (bx * fc) * dd(Sy, 0)
    if d3:
        p1y[i, j, k] = az * p1y[i, j, k] + (bz * fc) * dd(Sx, 2)
        p2x[i, j, k] = az * p2x[i, j, k] + (bz * fc) * dd(Sy, 2)
    p2y[i, j, k] = ax * p2y[i, j, k] + (bx * fc) * dd(Sz, 0)
    p2z[i, j, k] = ay * p2z[i, j, k] + (by * fc) * dd(Sx, 1)
    Dx, Dy, Dz = F[which + "x"], F[which + "y"], F[which + "z"]
    if which == "E":
        if d3:
            nx_ = ((Dx[i, j, k] + cy * dd(Sz, 1)) - cz * dd(Sy, 2)) + p1x[i, j, k] - p2x[i, j, k]
            ny_ = ((Dy[i, j, k] + cz * dd(Sx, 2)) - cx * dd(Sz, 0)) + p1y[i, j, k] - p2y[i, j, k]
        else:
            nx_ = (Dx[i, j, k] + cy * dd(Sz, 1)) + p1x[i, j, k]
            ny_ = (Dy[i, j, k] - cx * dd(Sz, 0)) - p2y[i, j, k]
        nz_ = ((Dz[i, j, k] + cx * dd(Sy, 0)) - cy * dd(Sx, 1)) + p1z[i, j, k] - p2z[i, j, k]
        xg, yg, zg = i + 1 - 3.0, j + 1 - 3.0, k + 1 - 3.0
        zero = [_beyond(prof, xg + 0.5, 0) | _beyond(prof, yg, 1) | _beyond(prof, zg, 2),
                _beyond(prof, xg, 0) | _beyond(prof, yg + 0.5, 1) | _beyond(prof, zg, 2),
                _beyond(prof, xg, 0) | _beyond(prof, yg, 1) | _beyond(prof, zg + 0.5, 2)]
    else:
        if d3:
            nx_ = ((Dx[i, j, k] - cy * dd(Sz, 1)) + cz * dd(Sy, 2)) - p1x[i, j, k] + p2x[i, j, k]
            ny_ = ((Dy[i, j, k] - cz * dd(Sx, 2)) + cx * dd(Sz, 0)) - p1y[i, j, k] + p2y[i, j, k]
        else:
            nx_ = (Dx[i, j, k] - cy * dd(Sz, 1)) - p1x[i, j, k]
            ny_ = (Dy[i, j, k] + cx * dd(Sz, 0)) + p2y[i, j, k]
        nz_ = ((Dz[i, j, k] - cx * dd(Sy, 0)) + cy * dd(Sx, 1)) - p1z[i, j, k] + p2z[i, j, k]
        xg, yg, zg = i + 1 - 3.0 + 0.5, j + 1 - 3.0 + 0.5, k + 1 - 3.0 + 0.5
        zero = [_beyond(prof, xg - 0.5, 0) | _beyond(prof, yg, 1) | _beyond(prof, zg, 2),
                _beyond(prof, xg, 0) | _beyond(prof, yg - 0.5, 1) | _beyond(prof, zg, 2),
                _beyond(prof, xg, 0) | _beyond(prof, yg, 1) | _beyond(prof, zg - 0.5, 2)]
    for D, v, z in ((Dx, nx_, zero[0]), (Dy, ny_, zero[1]), (Dz, nz_, zero[2])):
        D[i, j, k] = np.where(z, 0.0, v)


def _random_fields(g, seed):
    f = O.Fields(g)
    rng = np.random.default_rng(seed)
    for n in O.Fields.NAMES:
        getattr(f, n)[...] = rng.normal(size=O.grid_shape(g))
    return f


CASES = [
    (2, (30, 14, 1), {1: (4.0, 3.0), 2: (23.5, 4.0)}),
    (2, (24, 20, 1), {3: (2.2, 4.0), 4: (15.0, 2.0), 2: (18.0, 4.0)}),
    (3, (16, 12, 10), {1: (3.0, 2.5), 2: (11.0, 4.0), 5: (2.0, 3.0), 6: (6.5, 2.0)}),
]


@pytest.mark.parametrize("dims,n,faces", CASES)
def test_pml_matches_restatement(dims, n, faces):
    g = O.make_grid(dims, *n, c=0.45, qi=0.01)
    f = _random_fields(g, seed=17 + dims)
    pml = O.Pml(g, faces)
    o = O.Oracle(g, O.Particles(4), f.copy())
    F = {k: getattr(f, k).copy(order="F") for k in O.Fields.NAMES}
    psiE = [np.zeros(O.grid_shape(g), order="F") for _ in range(6)]
    psiB = [np.zeros(O.grid_shape(g), order="F") for _ in range(6)]
    for _ in range(2):
        o.pml_b(pml)
        _restated(g, F, psiB, faces, "B")
        o.pml_e(pml)
        _restated(g, F, psiE, faces, "E")
    for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        np.testing.assert_array_equal(getattr(o.f, k), F[k], err_msg=k)
    for a, b in zip(pml.psiE + pml.psiB, psiE + psiB):
        np.testing.assert_array_equal(a, b)
    # the interior box is untouched and its psi stays zero
    prof_ind = _profile(faces)[1]
    lo = [max(0, int(prof_ind[2 * a]) + 4) for a in range(3)]          # first 0-based index with g > ind(lo)
    hi = [min(O.grid_shape(g)[a], int(min(prof_ind[2 * a + 1], 1e6)) + 2) for a in range(3)]
    if dims == 2:
        lo[2], hi[2] = 0, 1
    box = tuple(slice(lo[a], hi[a]) for a in range(3))
    for k in ("Ex", "Bz"):
        np.testing.assert_array_equal(getattr(o.f, k)[box], getattr(f, k)[box])
    assert not pml.psiE[2][box].any()


def test_pml_no_faces_is_identity():
    g = O.make_grid(2, 16, 12, c=0.45, qi=0.01)
    f = _random_fields(g, seed=3)
    o = O.Oracle(g, O.Particles(4), f.copy())
    pml = O.Pml(g, {})
    o.pml_b(pml)
    o.pml_e(pml)
    for k in O.Fields.NAMES:
        np.testing.assert_array_equal(getattr(o.f, k), getattr(f, k))


def _pulse_energy(with_pml: bool, steps: int = 240):
    """A plane Ez/By pulse moving along +x in vacuum, stepped with the
    field phases in MAIN.F90 order (no particles); PML faces on both x
    sides when asked."""
    nx, ny = 96, 8
    g = O.make_grid(2, nx, ny, c=0.45, qi=0.01)
    f = O.Fields(g)
    x = np.arange(g.mx) - 3.0
    prof = np.exp(-((x - 40.0) / 5.0) ** 2)
    f.Ez[...] = prof[:, None, None]
    f.By[...] = -np.exp(-((x + 0.5 - 40.0) / 5.0) ** 2)[:, None, None]
    o = O.Oracle(g, O.Particles(4), f)
    pml = O.Pml(g, {1: (10.0, 8.0), 2: (85.0, 8.0)})
    e0 = o.field_energy()
    for _ in range(steps):
        o.update_b_half(); o.send_recv_flds("B")
        o.update_b_half()
        if with_pml:
            o.pml_b(pml)
        o.send_recv_flds("B")
        o.update_e()
        if with_pml:
            o.pml_e(pml)
        o.send_recv_flds("E")
    e = o.field_energy()
    return (e[0] + e[1]) / (e0[0] + e0[1])


def test_pml_absorbs_a_pulse():
    periodic = _pulse_energy(False)
    absorbed = _pulse_energy(True)
    assert abs(periodic - 1.0) < 0.02
    assert absorbed < 0.05
