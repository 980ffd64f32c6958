"""The oracle's field faces of EnforceBC_Final (src/bc/bc.F90:292-340) on
one rank against hand-derived answers: the 'attn' faces of
Attenuate_EM_Vacuum (a cubic ramp 1 - (d / scale)^3 beyond the face, cells
inside the face box untouched, diagonal cuts at the corners), the 'iflw'
face of Attenuate_EM_Flow (the layer relaxed towards the flow's -v x B and
B), and the 'open' x faces of OpenBC_Fld_Left/Right (halved components,
Bx copied from the face layer).  Global positions are local - 3 on one
rank."""
import numpy as np

from oracle import oracle as O


def _fields(g, seed=5):
    f = O.Fields(g)
    rng = np.random.default_rng(seed)
    for n in O.Fields.NAMES:
        getattr(f, n)[...] = rng.normal(size=O.grid_shape(g))
    return f


def _ramp(d, scale):
    return 1.0 - min(1.0, max(0.0, (abs(d) / scale) ** 3))


def test_attenuate_vacuum_one_face():
    g = O.make_grid(2, 12, 8, c=0.45, qi=0.01)          # mx = 17, my = 13
    f = _fields(g)
    F0 = {n: getattr(f, n).copy() for n in O.Fields.NAMES}
    o = O.Oracle(g, O.Particles(4), f)
    o.attenuate_vacuum({2: (5.0, 4.0)})                  # upper x face at x = 5, scale 4
    # attn_vac_pos_ind(2) = ceiling(5) + 1 = 6: cells with i - 3 < 6 (i <= 8) are left alone,
    # even where a component's staggered position lies beyond the face (Ex of i = 8 at x = 5.5)
    for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Jx", "Jy", "Jz"):
        np.testing.assert_array_equal(getattr(o.f, n)[:8], F0[n][:8], err_msg=n)
    for n in ("Jx", "Jy", "Jz"):
        np.testing.assert_array_equal(getattr(o.f, n), F0[n], err_msg=n)
    for i in range(9, g.mx + 1):                          # 1-based x index
        xi, xh = i - 3.0, i + 0.5 - 3.0
        for n, x in (("Ex", xh), ("Ey", xi), ("Ez", xi), ("Bx", xi), ("By", xh), ("Bz", xh)):
            np.testing.assert_array_equal(getattr(o.f, n)[i - 1], F0[n][i - 1] * _ramp(x - 5.0, 4.0), err_msg=n)
    assert o.f.Ex[8, 5, 0] == F0["Ex"][8, 5, 0] * (1.0 - (1.5 / 4.0) ** 3)   # i = 9: x = 6.5
    assert not o.f.Ey[11:].any()                          # x >= 9: (4 / 4)^3 = 1


def test_attenuate_vacuum_corner():
    """Two faces (upper x at 5, upper y at 3): beyond both, the x ramp holds
    while y <= 3 - 5 + x, the y ramp takes over above that diagonal."""
    g = O.make_grid(2, 12, 10, c=0.45, qi=0.01)
    f = O.Fields(g)
    f.Ey[...] = 1.0
    o = O.Oracle(g, O.Particles(4), f)
    o.attenuate_vacuum({2: (5.0, 4.0), 4: (3.0, 4.0)})
    # Ey at (i, j) lies at x = i - 3, y = j + 0.5 - 3
    i = 10                                                 # x = 7
    for j, expect in ((7, _ramp(2.0, 4.0)),                # y = 4.5 <= 5: x ramp
                      (8, _ramp(2.5, 4.0)),                # y = 5.5 > 5: y ramp, d = 2.5
                      (9, _ramp(3.5, 4.0))):               # y = 6.5: d = 3.5
        assert o.f.Ey[i - 1, j - 1, 0] == expect, (j, o.f.Ey[i - 1, j - 1, 0], expect)


def test_attenuate_flow():
    g = O.make_grid(2, 12, 8, c=0.45, qi=0.01)
    f = _fields(g, 7)
    F0 = {n: getattr(f, n).copy() for n in O.Fields.NAMES}
    b, v = (0.0, 0.0, 0.1), (-0.2, 0.0, 0.0)
    o = O.Oracle(g, O.Particles(4), f)
    o.attenuate_flow(2, 6.0, 2.0, 4.0, b, v)               # layer 4 <= x <= 6 beside the upper x face
    f0y = v[0] * b[2] - v[2] * b[0]                        # -0.02
    for i in range(1, g.mx + 1):
        x = i - 3.0
        inside = 4.0 <= x <= 6.0
        got, ref = o.f.Ey[i - 1], F0["Ey"][i - 1]
        if inside:
            np.testing.assert_array_equal(got, (ref - f0y) * _ramp(x - 6.0, 4.0) + f0y)
        else:
            np.testing.assert_array_equal(got, ref)
        xh = i + 0.5 - 3.0
        gotz, refz = o.f.Bz[i - 1], F0["Bz"][i - 1]
        if 4.0 <= xh <= 6.0:
            np.testing.assert_array_equal(gotz, (refz - b[2]) * _ramp(xh - 6.0, 4.0) + b[2])
        else:
            np.testing.assert_array_equal(gotz, refz)


def test_open_field_faces():
    g = O.make_grid(2, 12, 8, c=0.45, qi=0.01)
    f = _fields(g, 9)
    F0 = {n: getattr(f, n).copy() for n in O.Fields.NAMES}
    o = O.Oracle(g, O.Particles(4), f)
    o.open_fld_x(1, 6.2)                                    # xind_local = ceiling(9.2) = 10
    for n in ("Ey", "Ez"):
        np.testing.assert_array_equal(getattr(o.f, n)[:10], F0[n][:10])
        np.testing.assert_array_equal(getattr(o.f, n)[10:], 0.5 * F0[n][10:])
    for n in ("Ex", "By", "Bz"):
        np.testing.assert_array_equal(getattr(o.f, n)[:9], F0[n][:9])
        np.testing.assert_array_equal(getattr(o.f, n)[9:], 0.5 * F0[n][9:])
    np.testing.assert_array_equal(o.f.Bx[:10], F0["Bx"][:10])
    for i in range(10, g.mx):
        np.testing.assert_array_equal(o.f.Bx[i], F0["Bx"][9])
    f = _fields(g, 11)
    F0 = {n: getattr(f, n).copy() for n in O.Fields.NAMES}
    o = O.Oracle(g, O.Particles(4), f)
    o.open_fld_x(0, 1.0)                                    # xind_local = 4: layers 1..3
    for n in ("Ex", "Ey", "Ez", "By", "Bz"):
        np.testing.assert_array_equal(getattr(o.f, n)[:3], 0.5 * F0[n][:3])
        np.testing.assert_array_equal(getattr(o.f, n)[3:], F0[n][3:])
    for i in range(3):
        np.testing.assert_array_equal(o.f.Bx[i], F0["Bx"][3])


def test_open_particle_face_right():
    """OpenBC_Prtl_Right at x = 6 (local 9): the particle beyond becomes a
    hole, the ones in (8, 9) are mirrored to 18 - x and appended in slot
    order with u - gamma v0, v0 = the column's summed x velocity over
    1 + its count of flavours 1, 2, taken <= 0."""
    g = O.make_grid(2, 12, 8, c=0.45, qi=0.01)
    p = O.Particles(16)
    rows = [  # x, y, u, v, flv
        (9.5, 5.5, 0.2, 0.0, 1),    # beyond: hole
        (8.5, 5.5, 0.3, 0.1, 1),    # layer, column j = 5
        (8.2, 5.7, 0.1, 0.0, 2),    # layer, column j = 5
        (8.7, 6.2, -0.2, 0.05, 1),  # layer, column j = 6
        (7.5, 6.2, -0.4, 0.0, 1),   # inside, not in the layer
        (8.9, 6.8, -0.3, 0.0, 3),   # layer, column j = 6, flavour 3: mirrored, not averaged
    ]
    for n, (x, y, u, v, fl) in enumerate(rows):
        p.x[n], p.y[n], p.z[n], p.u[n], p.v[n], p.w[n], p.q[n], p.flv[n] = x, y, 1.5, u, v, 0.0, 1.0, fl
    p.used = len(rows)
    o = O.Oracle(g, p)
    assert o.open_prtl_x(1, 6.0) == 0
    v = o.p.view()
    assert o.p.used == len(rows) + 4
    assert v["flv"][0] == 0 and v["q"][0] == 0.0 and v["x"][0] == 3.8
    g5 = [np.sqrt(1.0 + 0.3 * 0.3 + 0.1 * 0.1 + 0.0), np.sqrt(1.0 + 0.1 * 0.1 + 0.0 + 0.0)]
    vel5 = ((0.0 + 0.3 * (1.0 / g5[0])) + 0.1 * (1.0 / g5[1])) / 3.0
    assert vel5 > 0                                   # taken as 0 on the right face
    g6 = np.sqrt(1.0 + 0.2 * 0.2 + 0.05 * 0.05 + 0.0)
    vel6 = (0.0 + -0.2 * (1.0 / g6)) / 2.0           # the flavour-3 particle is not averaged
    new = {k: a[len(rows):] for k, a in v.items()}
    np.testing.assert_array_equal(new["x"], [18.0 - 8.5, 18.0 - 8.2, 18.0 - 8.7, 18.0 - 8.9])
    np.testing.assert_array_equal(new["y"], [5.5, 5.7, 6.2, 6.8])
    np.testing.assert_array_equal(new["flv"], [1, 2, 1, 3])
    np.testing.assert_array_equal(new["u"][:2], [0.3, 0.1])
    np.testing.assert_array_equal(new["u"][2], -0.2 - g6 * vel6)
    np.testing.assert_array_equal(new["u"][3], -0.3 - np.sqrt(1.0 + 0.3 * 0.3 + 0.0 + 0.0) * vel6)
    np.testing.assert_array_equal(v["x"][1:6], [8.5, 8.2, 8.7, 7.5, 8.9])   # the originals stay


def test_open_particle_face_left_and_capacity():
    g = O.make_grid(2, 12, 8, c=0.45, qi=0.01)
    p = O.Particles(3)
    for n, (x, u) in enumerate(((3.5, 0.2), (4.6, 0.4))):   # face at 0.8 (local 3.8): hole, layer
        p.x[n], p.y[n], p.z[n], p.u[n], p.q[n], p.flv[n] = x, 5.5, 1.5, u, 1.0, 1
    p.used = 2
    o = O.Oracle(g, p)
    assert o.open_prtl_x(0, 0.8) == 0
    v = o.p.view()
    assert o.p.used == 3 and v["flv"][0] == 0
    ga = np.sqrt(1.0 + 0.4 * 0.4 + 0.0 + 0.0)
    vel = (0.0 + 0.4 * (1.0 / ga)) / 2.0             # >= 0 kept on the left face
    assert v["x"][2] == 2 * 3.8 - 4.6 and v["u"][2] == 0.4 - ga * vel
    # no room for another copy of the layer's two particles (capacity 3)
    assert o.open_prtl_x(0, 0.8) == -1
