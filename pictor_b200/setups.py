"""Synthetic initial conditions generated on the host (seeded), in the
reference layout that pic_load_particles takes.

``cyl_wakefield``: the cylindrical wakefield run.  A uniform electron plasma
loaded with even separation, npr x npt x npz particles per cell, weights
proportional to r (InitPrtlFromPSP_UniformSeparation, init_prtl.F90:224-352,
with azimuthal_weight_prtl, cyl_common.F90:57-62: weight = density * r * dtheta
per particle, so the charge per unit volume is npr*npt*npz * density), an
isotropic thermal spread, and a Gaussian electron bunch on the axis moving
along +z with Lorentz factor gamma.  The ions are an immobile neutralising
background (no ion particles; the initial E is zero).  Positions follow the
reference's cylindrical coordinates: x is r in cells shifted by 3 - rshift
(r = x - 3 + rmin with rmin = -0.5 on the rank holding the axis), y is theta
in cells (theta = (y - 3) * dtheta), z in cells.  Momenta are gamma*v in grid
units (the mover's gamma is sqrt(1 + |u|^2 / c^2), c the Courant number), so a
spread or a Lorentz factor given in units of the speed of light is scaled by c.
"""
from __future__ import annotations

import math

import numpy as np

from .simulation import Particles


def cyl_wakefield(nr: int, nz: int, ntheta: int, c: float, ppc=(2, 2, 2), density: float = 1.0, thermal: float = 0.01,
                  bunch_sigma_r: float = 20.0, bunch_sigma_z: float = 40.0, bunch_z0: float | None = None,
                  bunch_gamma: float = 50.0, bunch_peak: float = 0.1, bunch_particles: int = 1 << 18,
                  seed: int = 2930, rmin: float = -0.5) -> tuple[Particles, dict]:
    """Background electrons (flavour 2, charge -1 per unit weight) and bunch
    electrons (flavour 2); returns the particles and a summary.  ``thermal``
    is the per-component spread of gamma*beta; lengths are in cells."""
    rng = np.random.Generator(np.random.Philox(key=seed))
    dtheta = 2.0 * math.pi / ntheta
    npr, npt, npz = ppc
    # even placement inside each interior cell (x, y, z in ghosted cell units)
    fr = (np.arange(npr) + 0.5) / npr
    ft = (np.arange(npt) + 0.5) / npt
    fz = (np.arange(npz) + 0.5) / npz
    xi = (3 + np.arange(nr))[:, None] + fr[None, :]
    yi = (3 + np.arange(ntheta))[:, None] + ft[None, :]
    zi = (3 + np.arange(nz))[:, None] + fz[None, :]
    X, Y, Z = np.meshgrid(xi.ravel(), yi.ravel(), zi.ravel(), indexing="ij")
    X, Y, Z = X.ravel(), Y.ravel(), Z.ravel()
    r = np.maximum(X - 3.0 + rmin, 0.0)
    keep = r > 0
    X, Y, Z, r = X[keep], Y[keep], Z[keep], r[keep]
    wt = density * r * dtheta
    n_bg = X.size
    ub = rng.normal(scale=thermal * c, size=(3, n_bg))
    # bunch: Gaussian in (x, y) across the axis and in z, uniform weight
    z0 = bunch_z0 if bunch_z0 is not None else 3.0 + min(nz / 2.0, 6.0 * bunch_sigma_z)
    bx = rng.normal(scale=bunch_sigma_r, size=bunch_particles)
    by = rng.normal(scale=bunch_sigma_r, size=bunch_particles)
    bz = rng.normal(loc=z0, scale=bunch_sigma_z, size=bunch_particles)
    rb = np.hypot(bx, by)
    th = np.mod(np.arctan2(by, bx), 2.0 * math.pi)
    inside = (rb < nr - 1.0) & (bz >= 3.0) & (bz < 3.0 + nz)
    rb, th, bz = rb[inside], th[inside], bz[inside]
    # peak bunch density = bunch_peak x background density (charge per unit volume)
    n_unit = npr * npt * npz * density
    total = bunch_peak * n_unit * (2.0 * math.pi) ** 1.5 * bunch_sigma_r ** 2 * bunch_sigma_z
    wb = np.full(rb.size, total / bunch_particles)
    uzb = c * math.sqrt(bunch_gamma * bunch_gamma - 1.0)
    xs = np.concatenate([X, rb + 3.0 - rmin])
    ys = np.concatenate([Y, 3.0 + th / dtheta])
    zs = np.concatenate([Z, bz])
    n = xs.size
    p = Particles(q=-np.concatenate([wt, wb]), x=xs, y=ys, z=zs,
                  u=np.concatenate([ub[0], np.zeros(rb.size)]), v=np.concatenate([ub[1], np.zeros(rb.size)]),
                  w=np.concatenate([ub[2], np.full(rb.size, uzb)]), flv=np.full(n, 2, dtype=np.int32))
    return p, {"background": n_bg, "bunch": int(rb.size), "dtheta": dtheta, "bunch_z0": z0}
