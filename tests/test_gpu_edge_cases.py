"""Edge cases of the particle side on the GPU against the oracle's: a run
with no particles evolves the fields as in vacuum (J stays zero), and an
array of holes moves nothing, deposits nothing, appends nothing and
reorders to empty, in the FP64 form (fields bit for bit the oracle's) and
the FP32 form (fields to FP32 rounding); and a single particle, the
smallest ragged set, steps as the oracle's does."""
import numpy as np
import pytest

from oracle import oracle as O

from ._util import grid_and_config, random_fields, to_gpu_fields, to_gpu_particles

pytestmark = pytest.mark.gpu

NAMES6 = ("Ex", "Ey", "Ez", "Bx", "By", "Bz")


def _holes(g, n):
    return O.Particles.from_arrays(n + 8, q=np.zeros(n), x=np.full(n, 3.8), y=np.full(n, 3.8),
                                   z=np.full(n, 3.8 if g.dims == 3 else 1.5), u=np.zeros(n), v=np.zeros(n),
                                   w=np.zeros(n), flv=np.zeros(n, dtype=np.int32))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("kind", ["empty", "holes"])
def test_empty_and_all_hole_particle_sets(precision, dims, kind):
    from pictor_b200 import Simulation

    nx, ny, nz = (12, 10, 1) if dims == 2 else (8, 8, 8)
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, precision=precision, capacity=256, reorder_period=1)
    f = random_fields(g, seed=81, scale=0.05)
    o = O.Oracle(g, O.Particles(4), f.copy())
    for t in range(1, 4):
        assert o.step(t, 1) == 0
    assert not o.f.Jx.any() and o.p.used == 0
    p = O.Particles(4) if kind == "empty" else _holes(g, 64)
    with Simulation(cfg) as s:
        s.load_fields(to_gpu_fields(f))
        s.load_particles(to_gpu_particles(p))
        s.step(3)
        assert s.device_errors() == 0
        assert s.particle_count() == 0
        gf = s.fetch_fields()
    for n in ("Jx", "Jy", "Jz"):
        assert not getattr(gf, n).any(), n
    for n in NAMES6:
        a, b = getattr(gf, n), getattr(o.f, n)
        if precision == "fp64":
            np.testing.assert_array_equal(a, b, err_msg=n)
        else:
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-6 * np.abs(b).max(), err_msg=n)


@pytest.mark.parametrize("dims", [2, 3])
def test_single_particle_steps_as_oracle(dims):
    """One particle (every vector load and tile of the kernels partial):
    five FP64 steps with a reorder at step 2 and 4 equal the oracle's."""
    from pictor_b200 import Simulation

    nx, ny, nz = (12, 10, 1) if dims == 2 else (8, 8, 8)
    g, cfg = grid_and_config(dims=dims, nx=nx, ny=ny, nz=nz, capacity=64, reorder_period=2)
    p = O.Particles.from_arrays(16, q=np.array([1.0]), x=np.array([5.3]), y=np.array([6.7]),
                                z=np.array([4.2 if dims == 3 else 1.5]), u=np.array([0.6]), v=np.array([-0.4]),
                                w=np.array([0.3]), flv=np.array([1], dtype=np.int32))
    o = O.Oracle(g, p.copy())
    with Simulation(cfg) as s:
        s.load_particles(to_gpu_particles(p))
        for t in range(1, 6):
            o.step(t, 2)
            s.step(1)
        assert s.device_errors() == 0
        gp, gf = s.fetch_particles(), s.fetch_fields(with_current=False)
    v = o.p.view()
    live = v["flv"] != 0
    assert np.array_equal(gp.flv[gp.flv != 0], v["flv"][live])
    for k in ("x", "y", "z", "u", "v", "w"):
        np.testing.assert_allclose(getattr(gp, k)[gp.flv != 0], v[k][live], rtol=1e-12, atol=1e-12, err_msg=k)
    for n in NAMES6:
        a, b = getattr(gf, n), getattr(o.f, n)
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * max(np.abs(b).max(), 1e-30), err_msg=n)
