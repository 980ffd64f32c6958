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


def test_persistent_step_matches_separate_steps():
    """pic_step_persistent (every phase of every run in one persistent
    launch per span, the runs' reorders in between) against the runs stepped
    one after the other, across reorders at different periods per run: the
    same particles per run and energies to FP32 summation-order noise."""
    runs = _runs()
    tunings = {(r.nx, r.ny, r.ppc): Tuning(reorder_period=p) for r, p in zip(runs, (5, 7, 20))}
    together, t1 = run_batched(runs, 23, "fp32", tunings, batched=True, persistent=True)
    alone, t2 = run_batched(runs, 23, "fp32", tunings, batched=False)
    for a, b in zip(together, alone):
        assert a["particles"] == b["particles"]
        np.testing.assert_allclose(a["kinetic"], b["kinetic"], rtol=1e-5)
        np.testing.assert_allclose(a["B2"] + a["E2"], b["B2"] + b["E2"], rtol=1e-3)
        assert a["gauss_linf"] < 1e-2
    assert t1["particle_steps"] == t2["particle_steps"]
    # one launch per span (spans end at steps 5, 7, 10, 14, 15, 20, 21, 23)
    # plus the reorders, against at least four per run and step one by one
    assert t1["launches"] < t2["launches"] // 4


def test_persistent_step_3d_matches_step():
    """Two 3D FP32 runs (Lehe and Yee solvers are separate template cases;
    here Yee) through the persistent kernel against pic_step of each."""
    from pictor_b200 import PicConfig, Simulation, init_scale
    from pictor_b200.simulation import step_many

    sc = init_scale(0.45, 2.0, 4)
    shapes = [(32, 16, 16), (24, 24, 8)]
    res = {}
    for mode in ("alone", "persistent"):
        sims = []
        for i, (nx, ny, nz) in enumerate(shapes):
            cfg = PicConfig(nx=nx, ny=ny, nz=nz, dims=3, c=0.45, qi=sc["qi"], precision="fp32",
                            capacity=int(2 * 4 * nx * ny * nz * 1.05) + 4096, reorder_period=10)
            s = Simulation(cfg)
            s.init_weibel(4, 0.5, 0.3, 0.0008, 0.0008, 2930 + i)
            s.reorder()
            sims.append(s)
        try:
            if mode == "alone":
                for s in sims:
                    s.step(15)
            else:
                step_many(sims, 15, persistent=True)
            res[mode] = [s.diagnostics(sc["masse"]) for s in sims]
        finally:
            for s in sims:
                s.close()
    for a, b in zip(res["persistent"], res["alone"]):
        np.testing.assert_allclose(a["kinetic"], b["kinetic"], rtol=1e-5)
        np.testing.assert_allclose(a["B2"] + a["E2"], b["B2"] + b["E2"], rtol=1e-3)


def test_persistent_wait_timeout_returns_error_and_gpu_stays_usable():
    """The bound on the persistent kernel's waits: with force_timeout the
    first mover item waits for a count nothing reaches; after spin_limit
    polls the kernel records the timeout, every CTA stops, and the call
    returns PIC_ERR_TIMEOUT.  The GPU then still runs a normal step."""
    import torch

    from pictor_b200 import PicError
    from pictor_b200.simulation import step_many

    runs = _runs()[:2]
    sims = [make_run(r, "fp32") for r in runs]
    try:
        with pytest.raises(PicError) as e:
            step_many([s for s, _ in sims], 3, persistent=True, spin_limit=2000, force_timeout=True)
        assert e.value.code == -5
        torch.cuda.synchronize()
    finally:
        for s, _ in sims:
            s.close()
    # a fresh run steps normally afterwards
    sim, sc = make_run(runs[0], "fp32")
    with sim:
        sim.step(3)
        assert np.isfinite(sim.diagnostics(sc["masse"])["kinetic"]).all()
