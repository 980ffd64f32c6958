"""Ensembles of independent PIC runs (the batched form of the step).

An ensemble is a list of independent periodic runs of uneven grid size,
particles per cell, drift and temperature.  Across GPUs the runs shard with no
collective while stepping: ``partition`` assigns runs to ranks balanced by
particles x steps (largest-first greedy), each rank steps its own runs, and
``gather`` collects the per-run diagnostics on every rank at the end (the only
collective).  ``ensemble_runs`` draws the 64-run Weibel ensemble: per run r the
seed is 2930 + r (the reference's first seed word, initialise.F90:174).
"""
from __future__ import annotations

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

