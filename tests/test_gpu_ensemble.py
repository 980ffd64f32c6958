"""The batched form of the step on the GPU: pic_step_many against pic_step of
each run alone, the FP32 brick-shape override, and the per-size-class
autotuner."""
import numpy as np
import pytest

from pictor_b200.ensemble import RunSpec, Tuning, brick_candidates, make_run, run_batched, tune

pytestmark = pytest.mark.gpu


def _runs():
    # uneven sizes and fills, as in the 64-run ensemble
    return [RunSpec(run=0, nx=64, ny=64, ppc=4, drift=0.3, sigma=0.03, steps=12, seed=2930),
            RunSpec(run=1, nx=32, ny=48, ppc=8, drift=0.6, sigma=0.05, steps=12, seed=2931),
            RunSpec(run=2, nx=48, ny=32, ppc=16, drift=0.2, sigma=0.02, steps=12, seed=2932)]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_step_many_matches_separate_steps(precision):
    """Interleaving the runs' step graphs on their own streams changes
    nothing but the order of atomic sums: energies agree with the runs
    stepped one after the other (FP64 to 1e-10, FP32 to 1e-5)."""
    runs = _runs()
    together, t1 = run_batched(runs, 12, precision, batched=True)
    alone, t2 = run_batched(runs, 12, precision, batched=False)
    rtol = 1e-10 if precision == "fp64" else 1e-5
    for a, b in zip(together, alone):
        assert a["particles"] == b["particles"]
        np.testing.assert_allclose(a["kinetic"], b["kinetic"], rtol=rtol)
        np.testing.assert_allclose(a["B2"] + a["E2"], b["B2"] + b["E2"], rtol=100 * rtol)
    assert t1["particle_steps"] == t2["particle_steps"]


def test_one_launch_per_phase_matches_separate_steps():
    """pic_step_batched (every phase of a group of runs in one launch, the
    runs' reorders in between) against the runs stepped one after the other:
    the same particles per run and energies to FP32 summation-order noise."""
    runs = _runs()
    together, t1 = run_batched(runs, 12, "fp32", batched=True, per_phase=True)
    alone, t2 = run_batched(runs, 12, "fp32", batched=False)
    for a, b in zip(together, alone):
        assert a["particles"] == b["particles"]
        np.testing.assert_allclose(a["kinetic"], b["kinetic"], rtol=1e-5)
        np.testing.assert_allclose(a["B2"] + a["E2"], b["B2"] + b["E2"], rtol=1e-3)
    # four launches per group (at most four groups) and step; no reorder is due in 12 steps
    assert t1["launches"] == 4 * min(len(runs), 4) * 12


def test_brick_override_keeps_the_physics():
    """A requested brick shape changes how particles are grouped, not the
    step: energies after 10 steps match the automatic shape."""
    spec = _runs()[0]
    res = {}
    for brick in [(0, 0, 0), (16, 16, 1), (8, 8, 1)]:
        sim, sc = make_run(spec, "fp32", Tuning(brick=brick, reorder_period=5))
        with sim:
            sim.step(10)
            d = sim.diagnostics(sc["masse"])
        res[brick] = d
    ref = res[(0, 0, 0)]
    for brick, d in res.items():
        np.testing.assert_allclose(d["kinetic"], ref["kinetic"], rtol=1e-5, err_msg=str(brick))


def test_brick_too_large_is_rejected():
    from pictor_b200 import PicConfig, PicError, Simulation

    cfg = PicConfig(nx=256, ny=256, dims=2, precision="fp32", capacity=1 << 16, brick=(128, 128, 1))
    with pytest.raises(PicError) as e:
        Simulation(cfg)
    assert e.value.code == -1


def test_tuner_picks_a_candidate():
    spec = _runs()[2]
    t = tune(spec, periods=(5, 10), warmup=2)
    assert t.brick in brick_candidates(spec)
    assert t.reorder_period in (5, 10)
