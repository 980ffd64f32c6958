"""Ensembles of independent PIC runs (the batched form of the step).

An ensemble is a list of independent periodic runs of uneven grid size,
particles per cell, drift and temperature.  Across GPUs the runs shard with no
collective while stepping: ``partition`` assigns runs to ranks balanced by
particles x steps (largest-first greedy), each rank steps its own runs, and
``gather`` collects the per-run diagnostics on every rank at the end (the only
collective).  ``ensemble_runs`` draws the 64-run Weibel ensemble: per run r the
seed is 2930 + r (the reference's first seed word, initialise.F90:174).

On one GPU the runs of a rank step together: ``run_batched`` creates every
run, then ``step_many`` (pic_step_many) enqueues their step graphs
interleaved on one stream per run, so the small runs fill the GPU together.
``tune`` is the autotuner: per size class (grid, particles per cell) it times
a few candidate brick shapes and reorder periods on one run of the class and
keeps the fastest.
"""
from __future__ import annotations

import time
from dataclasses import asdict, dataclass

import numpy as np


@dataclass
class RunSpec:
    run: int
    nx: int
    ny: int
    ppc: int            # particles per cell per species
    drift: float        # beam speed / c along x
    sigma: float        # thermal spread / c  (Temp = 2 sigma^2)
    steps: int
    seed: int
    c: float = 0.45
    c_ompe: float = 2.0

    @property
    def temp(self) -> float:
        return 2.0 * self.sigma * self.sigma

    @property
    def particles(self) -> int:
        return 2 * self.ppc * self.nx * self.ny

    @property
    def cost(self) -> float:
        return float(self.particles) * self.steps


def ensemble_runs(n: int = 64, steps: int = 500, base_seed: int = 2930,
                  grids=(64, 128, 256, 512), ppcs=(4, 8, 16, 32)) -> list[RunSpec]:
    """The batched Weibel ensemble: grid uniform over `grids` (square), ppc
    uniform over `ppcs`, drift U(0.1, 0.9) c, spread U(0.01, 0.1) c."""
    runs = []
    for r in range(n):
        rng = np.random.Generator(np.random.Philox(key=base_seed + r))
        g = int(rng.choice(grids))
        runs.append(RunSpec(run=r, nx=g, ny=g, ppc=int(rng.choice(ppcs)), drift=float(rng.uniform(0.1, 0.9)),
                            sigma=float(rng.uniform(0.01, 0.1)), steps=steps, seed=base_seed + r))
    return runs


def partition(runs: list[RunSpec], world_size: int) -> list[list[int]]:
    """Largest-cost-first greedy assignment of runs to ranks; deterministic
    (ties broken by run index), so every rank computes the same plan."""
    order = sorted(range(len(runs)), key=lambda i: (-runs[i].cost, runs[i].run))
    load = [0.0] * world_size
    plan: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        plan[r].append(i)
        load[r] += runs[i].cost
    for p in plan:
        p.sort()
    return plan


def imbalance(runs: list[RunSpec], plan: list[list[int]]) -> float:
    loads = [sum(runs[i].cost for i in p) for p in plan]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def step_run(spec: RunSpec, precision: str = "fp32") -> dict:
    """Run one ensemble member on the current CUDA device; returns its
    diagnostics and particle count."""
    from .simulation import PicConfig, Simulation, init_scale

    sc = init_scale(spec.c, spec.c_ompe, spec.ppc)
    cap = int(spec.particles * 1.05) + 4096
    cfg = PicConfig(nx=spec.nx, ny=spec.ny, dims=2, c=spec.c, qi=sc["qi"], precision=precision, capacity=cap)
    with Simulation(cfg) as s:
        n = s.init_weibel(spec.ppc, 0.5, spec.drift, spec.temp, spec.temp, spec.seed)
        s.reorder()
        s.step(spec.steps)
        d = s.diagnostics(sc["masse"])
    return {"run": spec.run, "particles": n, "B2": float(d["B2"]), "E2": float(d["E2"]),
            "kinetic": [float(x) for x in d["kinetic"]], "gauss_linf": float(d["gauss_linf"])}


def gather(results: list[dict], world_size: int) -> list[dict]:
    """All-gather the per-run results of every rank (host objects); sorted by run."""
    if world_size == 1:
        return sorted(results, key=lambda d: d["run"])
    import torch.distributed as dist

    out: list = [None] * world_size
    dist.all_gather_object(out, results)
    merged = [d for part in out for d in part]
    return sorted(merged, key=lambda d: d["run"])


def run_ensemble(runs: list[RunSpec], rank: int, world_size: int, runner=step_run) -> list[dict]:
    """Each rank steps its share of the runs, then all results are gathered."""
    plan = partition(runs, world_size)
    mine = [runner(runs[i]) for i in plan[rank]]
    return gather(mine, world_size)


def as_dicts(runs: list[RunSpec]) -> list[dict]:
    return [asdict(r) for r in runs]



# ---------------------------------------------------------------------------
# Batched stepping on one GPU and the per-size-class autotuner
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class Tuning:
    brick: tuple = (0, 0, 0)      # FP32 brick shape, (0, 0, 0) = from the fill
    reorder_period: int = 20


def size_class(spec: RunSpec) -> tuple:
    return (spec.nx, spec.ny, spec.ppc)


def make_run(spec: RunSpec, precision: str = "fp32", tuning: Tuning | None = None):
    """Create and load one ensemble member (Weibel beams along x, Philox seed
    of the run); returns (Simulation, init_scale dict)."""
    from .simulation import PicConfig, Simulation, init_scale

    t = tuning or Tuning()
    sc = init_scale(spec.c, spec.c_ompe, spec.ppc)
    # the FP32 form wraps in place; the FP64 form keeps leavers as holes and
    # appends them until the next reorder, so it takes the reference's slack
    # (prtl_arr_size >= 3 * particles, initialise.F90:56-65)
    cap = int(spec.particles * (1.05 if precision == "fp32" else 3.0)) + 4096
    cfg = PicConfig(nx=spec.nx, ny=spec.ny, dims=2, c=spec.c, qi=sc["qi"], precision=precision, capacity=cap,
                    reorder_period=t.reorder_period, brick=t.brick if precision == "fp32" else (0, 0, 0))
    sim = Simulation(cfg)
    sim.init_weibel(spec.ppc, 0.5, spec.drift, spec.temp, spec.temp, spec.seed)
    sim.reorder()
    return sim, sc


def brick_candidates(spec: RunSpec) -> list[tuple]:
    """2D brick shapes holding between 1024 and 16384 particles at the run's
    fill (particles per cell = 2 ppc)."""
    shapes = [(8, 8, 1), (16, 8, 1), (16, 16, 1), (32, 16, 1), (32, 32, 1)]
    fill = 2 * spec.ppc
    out = [t for t in shapes if 1024 <= t[0] * t[1] * fill <= 16384 and t[0] <= spec.nx and t[1] <= spec.ny]
    return out or [(0, 0, 0)]


def _time_steps(sim, nsteps: int) -> float:
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim.step(nsteps)
    torch.cuda.synchronize()
    return time.perf_counter() - t0


def tune(spec: RunSpec, periods=(10, 20, 40), warmup: int = 3) -> Tuning:
    """Fastest (brick, reorder period) for the size class of `spec`: each
    candidate runs `warmup` steps, then 2 x period steps (two reorders) are
    timed; the measure is particle-steps per second."""
    best, best_rate = Tuning(), -1.0
    for brick in brick_candidates(spec):
        for period in periods:
            t = Tuning(brick=brick, reorder_period=period)
            sim, _ = make_run(spec, "fp32", t)
            try:
                sim.step(warmup)
                n = 2 * period
                rate = sim.particle_count() * n / _time_steps(sim, n)
            finally:
                sim.close()
            if rate > best_rate:
                best, best_rate = t, rate
    return best


def tune_classes(runs: list[RunSpec], **kw) -> dict:
    """Tuning per size class, each tuned on the class's first run."""
    out = {}
    for spec in runs:
        key = size_class(spec)
        if key not in out:
            out[key] = tune(spec, **kw)
    return out


def _diag(spec, sim, sc, n) -> dict:
    d = sim.diagnostics(sc["masse"])
    return {"run": spec.run, "particles": n, "B2": float(d["B2"]), "E2": float(d["E2"]),
            "kinetic": [float(x) for x in d["kinetic"]], "gauss_linf": float(d["gauss_linf"])}


def run_batched(runs: list[RunSpec], steps: int, precision: str = "fp32", tunings: dict | None = None,
                batched: bool = True, per_phase: bool = False, horizon: int = 0,
                persistent: bool = False) -> tuple[list[dict], dict]:
    """Step every run of the list `steps` times on the current GPU, together
    (pic_step_many; with per_phase pic_step_batched: one launch per phase
    for each group of runs; with persistent pic_step_persistent: one
    persistent launch per span between reorders) or one after the other;
    returns the per-run
    diagnostics and the timing {seconds, particle_steps, value, launches}.
    horizon > steps (together only): the runs then continue, untimed, to
    step `horizon`, and the timing dict carries their diagnostics there
    ("horizon")."""
    import torch

    from .simulation import step_many

    if not batched:
        return _run_one_by_one(runs, steps, precision, tunings)
    sims = []
    try:
        for spec in runs:
            t = (tunings or {}).get(size_class(spec))
            sims.append(make_run(spec, precision, t))
        counts = [s.particle_count() for s, _ in sims]
        for s, _ in sims:
            s.launch_count()   # reset the per-handle kernel counters
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        step_many([s for s, _ in sims], steps, per_phase=per_phase, persistent=persistent)
        torch.cuda.synchronize()
        secs = time.perf_counter() - t0
        launches = sum(s.launch_count() for s, _ in sims)
        results = [_diag(spec, s, sc, n) for spec, (s, sc), n in zip(runs, sims, counts)]
        at_horizon = None
        if horizon > steps:
            step_many([s for s, _ in sims], horizon - steps, per_phase=per_phase, persistent=persistent)
            at_horizon = [_diag(spec, s, sc, n) for spec, (s, sc), n in zip(runs, sims, counts)]
    finally:
        for s, _ in sims:
            s.close()
    ps = float(sum(counts)) * steps
    out = {"seconds": secs, "particle_steps": ps, "value": ps / secs, "launches": launches}
    if at_horizon is not None:
        out["horizon"] = at_horizon
    return results, out


def _run_one_by_one(runs: list[RunSpec], steps: int, precision: str, tunings: dict | None):
    """The plain form: each run created, stepped with pic_step and destroyed
    in turn; the timing sums the stepping of the runs only."""
    import torch

    results, secs, ps, launches = [], 0.0, 0.0, 0
    for spec in runs:
        sim, sc = make_run(spec, precision, (tunings or {}).get(size_class(spec)))
        with sim:
            n = sim.particle_count()
            sim.launch_count()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sim.step(steps)
            torch.cuda.synchronize()
            secs += time.perf_counter() - t0
            launches += sim.launch_count()
            d = sim.diagnostics(sc["masse"])
        ps += float(n) * steps
        results.append({"run": spec.run, "particles": n, "B2": float(d["B2"]), "E2": float(d["E2"]),
                        "kinetic": [float(x) for x in d["kinetic"]], "gauss_linf": float(d["gauss_linf"])})
    return results, {"seconds": secs, "particle_steps": ps, "value": ps / secs, "launches": launches}
