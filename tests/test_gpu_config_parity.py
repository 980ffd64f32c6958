"""Parity at the sizes of the benchmark configurations, against the OpenMP
build of the CPU restatement in its exact order (each cell's current summed
in particle order: the serial build's result at any thread count).

* The 2D FP64 Weibel configuration at full size: 256 x 256 cells, 16
  particles per cell per species (2.1 M particles), drift 0.5, thermal 0.05.
  With the exact-order current the GPU run equals the oracle bit for bit
  after 1, 5 and 21 steps (a reorder at 20); with the atomic current the
  particles are bit-exact after the first step and J agrees to 1e-12 of its
  scale.
* The 3D FP32 configuration's physics on the reduced 64 x 32 x 32 box
  (drift 0.3, thermal 0.02, 8 particles per cell per species): the FP64 form
  bit for bit over 21 steps, and the FP32 cell-relative form against the
  oracle over the configuration's 200 steps, energies within the bounds
  stated in the test.

Both sides start from the oracle's particles (the device loader's sin/cos
round differently from libm's in the last bit)."""
import numpy as np
import pytest

from oracle import oracle as O

from ._util import to_gpu_particles

pytestmark = pytest.mark.gpu

NAMES = ("q", "x", "y", "z", "u", "v", "w")


def _setup(dims, nx, ny, nz, epc, drift, temp, precision="fp64", exact=1, period=20):
    from pictor_b200 import PicConfig, init_scale

    sc = init_scale(0.45, 2.0, epc)
    g = O.make_grid(dims, nx, ny, nz, c=0.45, qi=sc["qi"])
    p = O.load_weibel(dims, nx, ny, nz, epc=epc, drift=drift, temp=temp, seed=2930)
    cap = int(p.used * 1.3) + 4096
    cfg = PicConfig(nx=nx, ny=ny, nz=nz, dims=dims, c=0.45, qi=sc["qi"], precision=precision, capacity=cap,
                    reorder_period=period, exact_current=exact)
    return g, cfg, p, sc


def _assert_bit_exact(s, o):
    gp = s.fetch_particles()
    v = o.p.view()
    assert len(gp.x) == o.p.used
    for k in NAMES:
        bad = np.count_nonzero(getattr(gp, k) != v[k])
        assert bad == 0, f"{k}: {bad} particles differ"
    assert np.array_equal(gp.flv, v["flv"])
    gf = s.fetch_fields(with_current=False)
    for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        assert np.array_equal(getattr(gf, n), getattr(o.f, n)), n


def test_weibel2d_full_grid_exact_order():
    from pictor_b200 import Simulation

    g, cfg, p, _ = _setup(2, 256, 256, 1, 16, 0.5, 0.005)
    assert p.used > 2_000_000
    o = O.Oracle(g, p.copy(), openmp=True, exact_order=True)
    with Simulation(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        done = 0
        for upto in (1, 5, 21):
            for t in range(done + 1, upto + 1):
                o.step(t, 20)
            s.step(upto - done)
            done = upto
            _assert_bit_exact(s, o)
        assert s.device_errors() == 0


def test_weibel2d_full_grid_atomic_current():
    """The default (atomic) current on the full grid: one move bit-exact in
    positions and momenta, J to 1e-12 of its scale."""
    from pictor_b200 import Simulation

    g, cfg, p, _ = _setup(2, 256, 256, 1, 16, 0.5, 0.005, exact=0)
    o = O.Oracle(g, p.copy(), openmp=True, exact_order=True)
    with Simulation(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        o.move_deposit()
        s.move_deposit()
        gp = s.fetch_particles()
        v = o.p.view()
        for k in NAMES:
            assert np.array_equal(getattr(gp, k), v[k]), k
        gf = s.fetch_fields()
        for n in ("Jx", "Jy", "Jz"):
            a, b = getattr(gf, n), getattr(o.f, n)
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * np.abs(b).max(), err_msg=n)


def test_weibel3d_reduced_box_fp64_exact_order():
    from pictor_b200 import Simulation

    g, cfg, p, _ = _setup(3, 64, 32, 32, 8, 0.3, 8e-4)
    o = O.Oracle(g, p.copy(), openmp=True, exact_order=True)
    with Simulation(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        done = 0
        for upto in (1, 21):
            for t in range(done + 1, upto + 1):
                o.step(t, 20)
            s.step(upto - done)
            done = upto
            _assert_bit_exact(s, o)


def test_weibel3d_reduced_box_fp32_200_steps():
    """The FP32 cell-relative form against the FP64 oracle over the
    configuration's 200 steps (reorders every 20): total, kinetic and field
    energy each within 2e-5 of the oracle's at every 20th step (measured on
    a B200: 8.0e-6 total, 8.0e-6 kinetic, 7.9e-6 field; the FP32 currents sum
    in an order that varies from run to run)."""
    from pictor_b200 import Simulation

    g, cfg, p, sc = _setup(3, 64, 32, 32, 8, 0.3, 8e-4, precision="fp32", exact=0)
    o = O.Oracle(g, p.copy(), openmp=True, exact_order=True)
    masse = sc["masse"]
    worst = {"total": 0.0, "kinetic": 0.0, "field": 0.0}
    with Simulation(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        for blk in range(10):
            for t in range(20 * blk + 1, 20 * blk + 21):
                o.step(t, 20)
            s.step(20)
            d = s.diagnostics(masse)
            fe = 0.5 * (d["B2"] + d["E2"])
            ke = float(sum(d["kinetic"]))
            ob, oe = o.field_energy()
            ofe = 0.5 * (ob + oe)
            oke = float(sum(o.particle_energy(masse)))
            worst["field"] = max(worst["field"], abs(fe - ofe) / ofe)
            worst["kinetic"] = max(worst["kinetic"], abs(ke - oke) / oke)
            worst["total"] = max(worst["total"], abs((fe + ke) - (ofe + oke)) / (ofe + oke))
    print("FP32 vs FP64 oracle, 64x32x32, 200 steps, max relative differences:", worst)
    assert worst["total"] <= 2e-5 and worst["kinetic"] <= 2e-5 and worst["field"] <= 2e-5, worst
