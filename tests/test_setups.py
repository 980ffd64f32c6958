"""The host-side initial conditions of pictor_b200.setups (no GPU)."""
import math

import numpy as np

from pictor_b200.setups import cyl_wakefield


def test_cyl_wakefield_layout_and_normalisation():
    nr, nz, nt, c = 16, 48, 8, 0.3
    p, info = cyl_wakefield(nr, nz, nt, c, bunch_sigma_r=3.0, bunch_sigma_z=6.0, bunch_particles=1 << 14,
                            thermal=0.01, bunch_gamma=50.0, bunch_peak=0.1, seed=7)
    n_bg, n_b = info["background"], info["bunch"]
    assert len(p.x) == n_bg + n_b
    # 2x2x2 per cell; the sub-position behind the axis (r < 0) is dropped
    assert n_bg == 8 * nr * nt * nz - 4 * nt * nz
    assert np.all(p.flv == 2)
    # interior of the ghosted grid
    assert p.x.min() >= 3.0 and p.x.max() < 3.0 + nr
    assert p.y.min() >= 3.0 and p.y.max() < 3.0 + nt
    assert p.z.min() >= 3.0 and p.z.max() < 3.0 + nz
    # background weight = density * r * dtheta, r = x - 3 + rmin with rmin = -0.5
    r = p.x[:n_bg] - 3.0 - 0.5
    np.testing.assert_allclose(-p.q[:n_bg], r * 2 * math.pi / nt, rtol=1e-14)
    # charge of the background = 8 per unit volume over the cylinder, up to the axis cell
    vol = math.pi * (nr - 0.5) ** 2 * nz
    assert abs(-p.q[:n_bg].sum() / (8 * vol) - 1.0) < 1.0 / nr
    # bunch: gamma 50 along +z (u in units of c), total charge of the Gaussian
    gam = np.sqrt(1.0 + (p.u[n_bg:] ** 2 + p.v[n_bg:] ** 2 + p.w[n_bg:] ** 2) / c ** 2)
    np.testing.assert_allclose(gam, 50.0, rtol=1e-12)
    total = 0.1 * 8 * (2 * math.pi) ** 1.5 * 3.0 ** 2 * 6.0
    np.testing.assert_allclose(-p.q[n_bg:], total / (1 << 14), rtol=1e-14)
    # background spread 0.01 c per component
    assert abs(p.u[:n_bg].std() / (0.01 * c) - 1.0) < 0.05


def test_cyl_wakefield_is_seeded():
    a, _ = cyl_wakefield(8, 16, 8, 0.3, bunch_particles=256, seed=3)
    b, _ = cyl_wakefield(8, 16, 8, 0.3, bunch_particles=256, seed=3)
    for k in a.NAMES:
        assert np.array_equal(getattr(a, k), getattr(b, k))
