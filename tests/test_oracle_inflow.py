"""The oracle's particle injection at an 'iflw' face (InjectNewPrtl,
src/bc/bc_inflow.F90:134-256) against hand-derived answers: the trial
region of SetInjDomain, the trial positions from the Philox draws (pinned
to the published vectors elsewhere), acceptance only in the layer the flow
emptied in one step, one particle per species per accepted position in
species order, and a drifting Maxwellian (AddDriftVel) in the mean."""
import numpy as np

from oracle import oracle as O

SP = [(1, 1e-3, 1.0), (2, 1e-3, -1.0)]


def _u01(hi, lo):
    return float(((int(hi) << 32) | int(lo)) >> 11) * (1.0 / 9007199254740992.0)


def test_region_positions_and_order():
    g = O.make_grid(2, 32, 16, c=0.45, qi=0.01)
    p = O.Particles(20000)
    p.used = 0
    o = O.Oracle(g, p)
    # upper x face at x = 20, flow -0.3c, vmax 0.5: trials in local x [20 - 0.225 + 3, 20 + 3)
    n = o.inject(2, 20.0, SP, epc=2000.0, density=1.0, drift=(-0.3, 0.0, 0.0), vmax=0.5, seed=7, call=3)
    v = o.p.view()
    assert n == o.p.used and n > 0 and n % 2 == 0
    x1, x2 = 20.0 - 0.5 * 0.45 + 3, 20.0 + 3
    front = 20.0 + (-0.3) * 0.45 + 3                     # accepted only at x >= pos + vx c
    assert (v["x"] >= front).all() and (v["x"] < x2).all()
    assert (v["y"] >= 3.0).all() and (v["y"] < 19.0).all() and (v["z"] >= 1.0).all() and (v["z"] < 2.0).all()
    np.testing.assert_array_equal(v["flv"], np.tile([1, 2], n // 2))
    np.testing.assert_array_equal(v["q"], np.tile([1.0, -1.0], n // 2))
    np.testing.assert_array_equal(v["x"][0::2], v["x"][1::2])   # both species at one position
    # the trial count is epc * volume = 2000 * 0.225 * 16 * 1 = 7200 (no Poisson draw above 1000); the
    # first accepted trial's position from its Philox draws
    key = (7, 0x494E4A43)
    for t in range(7200):
        r = O.philox((t, 3, 0, 0), key)
        r1, r2 = _u01(r[0], r[1]), _u01(r[2], r[3])
        r = O.philox((t, 3, 1, 0), key)
        racpt = _u01(r[2], r[3])
        xl = x1 + r1 * (x2 - x1)
        if racpt <= 1.0 and xl + (0.0 - 3.0) >= 20.0 + (-0.3) * 0.45:
            break
    assert v["x"][0] == xl and v["y"][0] == 3.0 + r2 * (19.0 - 3.0)
    # 0.135 / 0.225 of the trials fall in the emptied layer
    assert abs(n / 2 / 7200 - 0.6) < 0.03
    # the drift in the mean: u / gamma of a cold Maxwellian boosted by -0.3c
    gam = np.sqrt(1 + v["u"] ** 2 + v["v"] ** 2 + v["w"] ** 2)
    assert abs(np.mean(v["u"] / gam) + 0.3) < 0.01 and abs(np.mean(v["v"] / gam)) < 0.01


def test_lower_face_moving_injector_and_poisson_count():
    g = O.make_grid(2, 32, 16, c=0.45, qi=0.01)
    p = O.Particles(4000)
    p.used = 0
    o = O.Oracle(g, p)
    # lower x face at 10 moving at 0.5c, flow +0.2c: trials in [10 - 0.225, 10 + 0.45] (+3)
    n = o.inject(1, 10.0, SP[:1], epc=4.0, density=0.5, drift=(0.2, 0.0, 0.0), speed=0.5, vmax=1.0, seed=11, call=0)
    v = o.p.view()
    # 4 * 0.675 * 16 = 43.2 -> 43 trials, then a Poisson draw of mean 43; half accepted by the density,
    # and only x <= pos + vx c = 10.09 (global)
    assert 0 < n < 80
    assert (v["x"] >= 10.0 - 0.225 + 3).all() and (v["x"] <= 10.0 + 0.2 * 0.45 + 3).all()
    np.testing.assert_array_equal(v["flv"], np.ones(n, dtype=np.int32))
    # capacity: no room for a second injection of 4000 trials -> -1, nothing appended
    before = o.p.used
    assert o.inject(1, 10.0, SP, epc=4000.0, density=1.0, drift=(0.2, 0.0, 0.0), speed=0.5, seed=11, call=1) == -1
    assert o.p.used == before


def test_fluid_frame_reflection():
    """RefPrtlFluidFrameRight: a particle beyond the drifted injector layer
    is reflected in the flow's frame (for a flow at rest, u -> -u), mirrored
    across the layer, and the current of that move is the zigzag current of
    DepositCurrentPIC (here a move inside one cell: Jx(i, j) and Jx(i, j+1)
    share F = q qi dx in the ratio of the midpoint's y weight)."""
    g = O.make_grid(2, 32, 16, c=0.45, qi=0.01)
    p = O.Particles(4)
    rows = [(23.4, 7.25, 0.2, 1.0), (22.6, 7.5, 0.1, 1.0), (23.9, 8.5, -0.1, 0.0)]   # x, y, u, q
    for n, (x, y, u, q) in enumerate(rows):
        p.x[n], p.y[n], p.z[n], p.u[n], p.q[n], p.flv[n] = x, y, 1.5, u, q, (1 if q else 0)
    p.used = 3
    f = O.Fields(g)
    o = O.Oracle(g, p, f)
    o.reflect_fluid_right(20.0, 0.0)                     # layer at 23.0 (local), no flow
    v = o.p.view()
    assert v["x"][0] == 2.0 * 23.0 - 23.4 and v["u"][0] == -0.2
    assert v["x"][1] == 22.6 and v["u"][1] == 0.1          # before the layer: untouched
    assert v["x"][2] == 23.9                               # a hole (q = 0): untouched
    # the move 23.4 -> 22.6 crosses x = 23: two segments, Jx of cells 23 and 22 at y weights of 7.25
    F1, F2 = 0.01 * (23.0 - 23.4), 0.01 * (22.6 - 23.0)
    np.testing.assert_allclose(o.f.Jx[22, 6, 0], F1 * (1 - 0.25))
    np.testing.assert_allclose(o.f.Jx[22, 7, 0], F1 * 0.25)
    np.testing.assert_allclose(o.f.Jx[21, 6, 0], F2 * (1 - 0.25))
    np.testing.assert_allclose(o.f.Jx[21, 7, 0], F2 * 0.25)
    assert abs(o.f.Jx.sum() - 0.01 * (22.6 - 23.4)) < 1e-15
    # a flow drifting at -0.3c: u is reflected in the flow's frame (gamma-boosted), the layer at 23 - 0.135
    p = O.Particles(2)
    p.x[0], p.y[0], p.z[0], p.u[0], p.q[0], p.flv[0] = 23.2, 7.5, 1.5, -0.1, 1.0, 1
    p.used = 1
    o = O.Oracle(g, p, O.Fields(g))
    o.reflect_fluid_right(20.0, -0.3)
    dg, db = 1 / np.sqrt((1 + 0.3) * (1 - 0.3)), -0.3
    u = -0.1
    gam = np.sqrt(1 + u * u)
    u = -(dg * u + dg * (-db) * gam)
    gam = np.sqrt(1 + u * u)
    u = dg * u + dg * db * gam
    np.testing.assert_allclose(o.p.view()["u"][0], u, rtol=1e-15)
    assert o.p.view()["x"][0] == 2.0 * (23.0 - 0.3 * 0.45) - 23.2
