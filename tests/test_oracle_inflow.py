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
