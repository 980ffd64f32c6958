"""The oracle's walls along x (src/bc/bc_reflect.F90 on one rank) against
hand-derived answers: specular reflection of the particles beyond the wall,
the current beyond the wall folded back onto the first layer inside it
(tangential components added, the normal one subtracted), and the tangential
E zeroed beyond a conducting wall."""
import numpy as np

from oracle import oracle as O


def _state():
    g = O.make_grid(2, 12, 8, c=0.45, qi=0.01)
    p = O.Particles(16)
    xs = [4.2, 5.0, 3.8, 11.7, 11.4, 7.0]
    us = [-0.3, 0.1, 0.0, 0.2, 0.25, -0.1]
    flv = [1, 2, 0, 2, 1, 1]
    for n, (x, u, fl) in enumerate(zip(xs, us, flv)):
        p.x[n], p.u[n], p.flv[n] = x, u, fl
        p.y[n], p.z[n], p.q[n] = 5.5, 1.5, (1.0 if fl else 0.0)
    p.used = len(xs)
    f = O.Fields(g)
    rng = np.random.default_rng(3)
    for n in O.Fields.NAMES:
        getattr(f, n)[...] = rng.normal(size=O.grid_shape(g))
    return g, p, f


def test_reflecting_walls():
    g, p, f = _state()
    J0 = {n: getattr(f, n).copy() for n in ("Jx", "Jy", "Jz")}
    o = O.Oracle(g, p, f)
    o.reflect_particles_x(0, 1.5)     # wall at x = 4.5 (local)
    o.reflect_particles_x(1, 8.5)     # wall at x = 11.5
    v = o.p.view()
    np.testing.assert_array_equal(v["x"], [2.0 * 4.5 - 4.2, 5.0, 3.8, 2.0 * 11.5 - 11.7, 11.4, 7.0])
    np.testing.assert_array_equal(v["u"], [0.3, 0.1, 0.0, -0.2, 0.25, -0.1])
    # left: Jy, Jz layer 5 += layer 4 (ceiling(1.5 + 3)), Jx layer 4 -= layer 3 (ceiling(1.0 + 3))
    # right: Jy, Jz layer 11 += layer 12 (floor(8.5 + 3)), Jx layer 11 -= layer 12 (floor(8.0 + 3))
    ex = {n: a.copy() for n, a in J0.items()}
    for n in ("Jy", "Jz"):
        ex[n][4] = J0[n][4] + J0[n][3]
        ex[n][3] = 0.0
        ex[n][10] = J0[n][10] + J0[n][11]
        ex[n][11] = 0.0
    ex["Jx"][3] = J0["Jx"][3] - J0["Jx"][2]
    ex["Jx"][2] = 0.0
    ex["Jx"][10] = J0["Jx"][10] - J0["Jx"][11]
    ex["Jx"][11] = 0.0
    for n in ("Jx", "Jy", "Jz"):
        np.testing.assert_array_equal(getattr(o.f, n), ex[n], err_msg=n)


def test_conducting_walls():
    g, p, f = _state()
    E0 = {n: getattr(f, n).copy() for n in ("Ex", "Ey", "Ez")}
    o = O.Oracle(g, p, f)
    o.conducting_x(0, 1.5)            # layers 1..4 (floor(4.5))
    o.conducting_x(1, 8.5)            # layers 12..mx (ceiling(11.5))
    for n in ("Ey", "Ez"):
        a = getattr(o.f, n)
        assert not a[:4].any() and not a[11:].any()
        np.testing.assert_array_equal(a[4:11], E0[n][4:11])
    np.testing.assert_array_equal(o.f.Ex, E0["Ex"])


def test_y_walls():
    """Bottom wall at y = 4.5 (pos 1.5), top wall at y = 8.5 (pos 5.5) on
    a 12 x 8 grid (my = 13): W = int(4.5) = 4 and int(8.5) = 8."""
    g, p, f = _state()
    for n, y in enumerate([4.2, 5.0, 3.8, 8.7, 8.4, 6.0]):
        p.y[n], p.v[n] = y, [-0.3, 0.1, 0.0, 0.2, 0.25, -0.1][n]
    J0 = {n: getattr(f, n).copy() for n in ("Jx", "Jy", "Jz")}
    E0 = {n: getattr(f, n).copy() for n in ("Ex", "Ey", "Ez")}
    o = O.Oracle(g, p, f)
    o.reflect_particles_y(0, 1.5)
    o.reflect_particles_y(1, 5.5)
    v = o.p.view()
    np.testing.assert_array_equal(v["y"], [2.0 * 4.5 - 4.2, 5.0, 3.8, 2.0 * 8.5 - 8.7, 8.4, 6.0])
    np.testing.assert_array_equal(v["v"], [0.3, 0.1, 0.0, -0.2, 0.25, -0.1])
    ex = {n: a.copy() for n, a in J0.items()}
    # bottom (W = 4, 0-based 3): Jx, Jz += layer 3; Jy -= layer 3; layer 3 zeroed
    for n, sgn in (("Jx", 1), ("Jy", -1), ("Jz", 1)):
        ex[n][:, 3] = J0[n][:, 3] + sgn * J0[n][:, 2]
        ex[n][:, 2] = 0.0
    # top (W = 8, 0-based 7): Jx, Jz(8) += (9); Jy(7) -= Jy(8); Jx, Jz(9) and Jy(8) zeroed
    for n in ("Jx", "Jz"):
        ex[n][:, 7] = ex[n][:, 7] + ex[n][:, 8]
        ex[n][:, 8] = 0.0
    ex["Jy"][:, 6] = ex["Jy"][:, 6] - ex["Jy"][:, 7]
    ex["Jy"][:, 7] = 0.0
    for n in ("Jx", "Jy", "Jz"):
        np.testing.assert_array_equal(getattr(o.f, n), ex[n], err_msg=n)
    o.conducting_y(0, 1.5)            # y layers 1..4
    o.conducting_y(1, 5.5)            # y layers 9..13
    for n in ("Ex", "Ez"):
        a = getattr(o.f, n)
        assert not a[:, :4].any() and not a[:, 8:].any()
        np.testing.assert_array_equal(a[:, 4:8], E0[n][:, 4:8])
    np.testing.assert_array_equal(o.f.Ey, E0["Ey"])


def test_remove_beyond_walls():
    """RemovePrtl at the low x face (x < 4.5) and the high y face (y > 6.5):
    those particles become holes with RemovePrtl's values, the rest stay."""
    g, p, f = _state()
    for n, y in enumerate([5.0, 5.0, 3.8, 7.0, 5.5, 6.0]):
        p.y[n] = y
    o = O.Oracle(g, p, f)
    o.remove_particles(1, 1.5)
    o.remove_particles(4, 3.5)
    v = o.p.view()
    # particle 0 (x 4.2) and 3 (y 7.0) removed; 2 was a hole already
    np.testing.assert_array_equal(v["flv"], [0, 2, 0, 0, 1, 1])
    for n in (0, 3):
        assert (v["q"][n], v["u"][n], v["x"][n], v["y"][n], v["z"][n]) == (0.0, 0.0, 3.8, 3.8, 1.5)
    np.testing.assert_array_equal(v["x"][[1, 4, 5]], [5.0, 11.4, 7.0])
