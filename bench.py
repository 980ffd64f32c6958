"""Throughput of the PIC step on B200: particle-steps/s.

Default workload: the 3D Cartesian Weibel run in the FP32 cell-relative form
(512x256x256 cells, 8 particles per cell per species in two counter-streaming
e+- beams at +-0.3c, thermal spread 0.02c, Courant 0.45, periodic), with
synthetic inputs generated from Philox-4x32-10 on the device.  The same seed
is also stepped in the FP64 reference form; their throughput ratio and field
/ total energy difference are reported beside the headline.

One JSON line on stdout (rank 0).  Under torchrun every rank runs its own
replica (seed + rank): weak scaling with no data-path collective; the timed
region is bracketed by a barrier and the max over ranks is taken.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s on 1 B200 (FP32/batched vs plain FP64) at stated energy error"

WORKLOADS = {
    # configs: the 3D FP32 Weibel run (headline) and the 2D FP64 Weibel run
    "weibel3d_fp32": dict(dims=3, nx=512, ny=256, nz=256, epc=8, drift=0.3, temp=8e-4, c=0.45, c_ompe=2.0,
                          precision="fp32", horizon=200),
    "weibel2d_fp64": dict(dims=2, nx=256, ny=256, nz=1, epc=16, drift=0.5, temp=0.005, c=0.45, c_ompe=2.0,
                          precision="fp64", horizon=1000),
    # a small case of the headline physics for profiler captures (particles 270 MB > L2)
    "weibel3d_fp32_small": dict(dims=3, nx=128, ny=64, nz=64, epc=8, drift=0.3, temp=8e-4, c=0.45, c_ompe=2.0,
                                precision="fp32", horizon=200),
    # the same small case in the FP64 reference layout (the tiled FP64 mover)
    "weibel3d_fp64_small": dict(dims=3, nx=128, ny=64, nz=64, epc=8, drift=0.3, temp=8e-4, c=0.45, c_ompe=2.0,
                                precision="fp64", fp64_tiles=1),
    # the batched ensemble: 64 independent 2D Weibel runs, grid 64^2..512^2, 4..32 particles per cell per
    # species, drift U(0.1, 0.9) c, spread U(0.01, 0.1) c, seed 2930 + run (pictor_b200.ensemble)
    "ensemble64": dict(dims=2, runs=64, epc=16, drift=0.5, temp=0.005, c=0.45, c_ompe=2.0, precision="fp32",
                       nx=256, ny=256, nz=1, horizon=500),
    # the 2D FP64 Weibel configuration split along x into one slab per rank (strong scaling: the
    # global grid fixed), the slabs exchanging their x faces over NCCL between the phases
    "slab_weibel2d_fp64": dict(dims=2, nx=256, ny=256, nz=1, epc=16, drift=0.5, temp=0.005, c=0.45, c_ompe=2.0,
                               precision="fp64", cpu_workload="weibel2d_fp64"),
    # the 3D FP32 Weibel configuration (the headline's) split along x into one slab per rank
    "slab_weibel3d_fp32": dict(dims=3, nx=512, ny=256, nz=256, epc=8, drift=0.3, temp=8e-4, c=0.45, c_ompe=2.0,
                               precision="fp32", cpu_workload="weibel3d_fp32"),
    # the differentiable 2D Weibel run: 128^2 cells, 8 particles per cell per species, drift +-0.4c, spread
    # 0.05c, 400 steps, checkpoints every 50, objective sum_t 1/2 sum |B_t|^2 (pictor_b200.adjoint)
    "adjoint128": dict(dims=2, nx=128, ny=128, nz=1, epc=8, drift=0.4, temp=0.005, c=0.45, c_ompe=2.0,
                       precision="fp32", nsteps=400, checkpoint=50),
    # the cylindrical wakefield configuration in the reference's theta-gridded form (FP64, Lehe along z):
    # Nr = 256, Nz = 2048, 8 theta cells, dr = dz = 0.1 c/wp, 2x2x2 electrons per cell weighted by r with
    # 0.01c spread, neutralising ions, Gaussian bunch sigma_r = 2, sigma_z = 4 c/wp, gamma 50, 0.1 x n0;
    # Courant 0.3 (stable next to the axis with 8 theta cells)
    "cyl_wake": dict(dims=3, nx=256, ny=8, nz=2048, epc=8, c=0.3, c_ompe=10.0, precision="fp64", thermal=0.01,
                     bunch_gamma=50.0, bunch_peak=0.1, bunch_sigma_r=20.0, bunch_sigma_z=40.0),
    # the same run with the field solve on azimuthal modes m = 0, 1 (the theta-gridded scheme projected
    # onto them; particles gather from / deposit onto the 8 theta cells)
    "cyl_wake_modal": dict(dims=3, nx=256, ny=8, nz=2048, epc=8, c=0.3, c_ompe=10.0, precision="fp64", thermal=0.01,
                           bunch_gamma=50.0, bunch_peak=0.1, bunch_sigma_r=20.0, bunch_sigma_z=40.0, cyl_modes=2),
    # the same run in the FP32 cell-relative form (theta-gridded FP32 fields)
    "cyl_wake_fp32": dict(dims=3, nx=256, ny=8, nz=2048, epc=8, c=0.3, c_ompe=10.0, precision="fp32", thermal=0.01,
                          bunch_gamma=50.0, bunch_peak=0.1, bunch_sigma_r=20.0, bunch_sigma_z=40.0, horizon=2000),
    # the C3 configuration as stated: modes m = 0, 1, FP32 fields and particles
    "cyl_wake_modal_fp32": dict(dims=3, nx=256, ny=8, nz=2048, epc=8, c=0.3, c_ompe=10.0, precision="fp32",
                                thermal=0.01, bunch_gamma=50.0, bunch_peak=0.1, bunch_sigma_r=20.0, bunch_sigma_z=40.0,
                                cyl_modes=2, horizon=2000),
    # small cases of the same physics for profiler captures (4.2 M particles, 250 MB > L2)
    "cyl_wake_small_modal_fp32": dict(dims=3, nx=64, ny=8, nz=1024, epc=8, c=0.3, c_ompe=10.0, precision="fp32",
                                      thermal=0.01, bunch_gamma=50.0, bunch_peak=0.1, bunch_sigma_r=5.0,
                                      bunch_sigma_z=10.0, cyl_modes=2),
    "cyl_wake_small_fp32": dict(dims=3, nx=64, ny=8, nz=1024, epc=8, c=0.3, c_ompe=10.0, precision="fp32",
                                thermal=0.01, bunch_gamma=50.0, bunch_peak=0.1, bunch_sigma_r=5.0, bunch_sigma_z=10.0),
    "cyl_wake_small": dict(dims=3, nx=64, ny=8, nz=1024, epc=8, c=0.3, c_ompe=10.0, precision="fp64", thermal=0.01,
                           bunch_gamma=50.0, bunch_peak=0.1, bunch_sigma_r=5.0, bunch_sigma_z=10.0),
}
SEED = 2930


def bytes_per_particle(dims: int, precision: str) -> int:
    """Algorithmic bytes per particle-step: each SoA field read once and the
    updated ones written once."""
    if precision == "fp32":
        return 60 if dims == 3 else 52
    return 108


def bytes_per_cell_mover(precision: str) -> int:
    """Grid bytes of the mover per interior cell: gather of 6 field components
    + deposit of 3 current components."""
    return 9 * (4 if precision == "fp32" else 8)


# DRAM bytes (read + written) per particle of one k_move_f32_tiled<3> launch,
# from ncu (dram__bytes_read.sum + dram__bytes_write.sum) on the
# weibel3d_fp32_small workload (8.39 M particles, 270 MB of particle state,
# larger than L2); scaled to a full launch by the particles it moves.
TRAFFIC_BYTES_PER_PARTICLE = 57.1
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of k_move_f32_tiled on weibel3d_fp32_small, "
                  "per particle, scaled by the particles of the launch")


def traffic_per_launch(wl: dict, n_p: int):
    if wl["precision"] != "fp32" or wl["dims"] != 3:
        return None
    return TRAFFIC_BYTES_PER_PARTICLE * n_p


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.device = device
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus: int):
    import torch

    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(ws, value: float) -> float:
    if ws == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(ws, value: float) -> float:
    if ws == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def mover_kernel(wl: dict, precision: str) -> str:
    """The mover kernel of the timed steps (after a reorder): the FP32 tiled
    mover, or the FP64 one by tiles unless tiles are switched off."""
    if precision == "fp32":
        return "k_move_f32_tiled (timed with the k_node_avg pass it reads from)"
    return "k_move_f64" if wl.get("fp64_tiles", 0) < 0 else "k_move_f64_tiled"


def make_sim(wl: dict, precision: str, extra_capacity: float = 1.04):
    from pictor_b200 import PicConfig, Simulation, init_scale

    sc = init_scale(wl["c"], wl["c_ompe"], wl["epc"])
    vol = wl["nx"] * wl["ny"] * (wl["nz"] if wl["dims"] == 3 else 1)
    cap = int(2 * wl["epc"] * vol * extra_capacity) + (1 << 16)
    cfg = PicConfig(nx=wl["nx"], ny=wl["ny"], nz=wl["nz"], dims=wl["dims"], c=wl["c"], qi=sc["qi"],
                    precision=precision, capacity=cap, reorder_period=20, fp64_tiles=wl.get("fp64_tiles", 0))
    return Simulation(cfg), sc


def timed_steps(sim, steps: int, ws: int, profile: bool):
    """K steps bracketed by barrier + synchronize; CUDA events on the
    library's stream.  Returns (ms total, phase times, launches)."""
    import torch

    stream = torch.cuda.ExternalStream(sim.stream)
    sim.profile(profile)
    sim.phase_times()
    sim.launch_count()
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    ms = e0.elapsed_time(e1)
    phases = sim.phase_times() if profile else None
    launches = sim.launch_count()
    sim.profile(False)
    return ms, phases, launches


def energy_curve(sim, sc, done: int, horizon: int, every: int = 20) -> dict:
    """Step a run from step `done` to `horizon`, recording its energies at
    every multiple of `every` (and at the horizon)."""
    curve = {}
    t = done
    while t < horizon:
        nxt = min(horizon, (t // every + 1) * every)
        sim.step(nxt - t)
        t = nxt
        curve[t] = energies(sim, sc)
    return curve


def curve_errors(a: dict, b: dict) -> dict:
    """Max relative differences of curve a from curve b (FP64) over their
    common steps: field, kinetic and total energy; and the values at the last."""
    steps = sorted(set(a) & set(b))
    if not steps:
        return {}
    def rel(x, y):
        return abs(x - y) / max(abs(y), 1e-300)
    last = steps[-1]
    out = {"steps_compared": [steps[0], last], "points": len(steps),
           "field_energy_rel_err_max": max(rel(a[t]["field"], b[t]["field"]) for t in steps),
           "kinetic_energy_rel_err_max": max(rel(a[t]["kinetic"], b[t]["kinetic"]) for t in steps),
           "total_energy_rel_err_max": max(rel(a[t]["field"] + a[t]["kinetic"], b[t]["field"] + b[t]["kinetic"])
                                           for t in steps),
           "field_energy_at_horizon": {"fp32": a[last]["field"], "fp64": b[last]["field"]}}
    # the Gauss residual where the diagnostics form it (the Cartesian grid; rho_max 0 otherwise)
    if a[last]["rho_max"] > 0 and b[last]["rho_max"] > 0:
        out["gauss_linf_over_rho_at_horizon"] = {"fp32": a[last]["gauss_linf"] / a[last]["rho_max"],
                                                 "fp64": b[last]["gauss_linf"] / b[last]["rho_max"]}
    return out


def energies(sim, sc) -> dict:
    d = sim.diagnostics(sc["masse"])
    return {"field": 0.5 * (d["B2"] + d["E2"]), "B": 0.5 * d["B2"], "kinetic": float(sum(d["kinetic"])),
            "gauss_linf": d["gauss_linf"], "rho_max": d["rho_max"]}


def cpu_sample(wl: dict, target_s: float = 12.0, threads: int | None = None):
    """The reference CPU step (C restatement, OpenMP over 32-particle blocks
    as the reference's OPEN_MP build) on a bounded sub-box of the workload
    with the same physics; returns particle-steps/s and what was timed."""
    from oracle import oracle as O

    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    dims = wl["dims"]
    if dims == 3:
        nx, ny, nz = 96, 48, 48
    else:
        nx, ny, nz = 256, 256, 1
    qi = O.init_scale(wl["c"], wl["c_ompe"], wl["epc"])[0]
    g = O.make_grid(dims, nx, ny, nz, c=wl["c"], qi=qi)
    p = O.load_weibel(dims, nx, ny, nz, epc=wl["epc"], drift=wl["drift"], temp=wl["temp"], seed=SEED)
    o = O.Oracle(g, p, openmp=True, exact_order=False)   # the reference's thread slices
    o.step(1)
    n_steps, t0, t = 0, time.perf_counter(), 1
    while True:
        t += 1
        o.step(t)
        n_steps += 1
        el = time.perf_counter() - t0
        if el >= target_s or n_steps >= 200:
            break
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": p.used * n_steps / el, "unit": "particle-steps/s", "cores": cores, "kind": "port",
            "sample": f"{'x'.join(map(str, (nx, ny, nz)[:dims]))} cells, {p.used} particles, {n_steps} steps "
                      f"(same physics and seed), FP64, C restatement of the reference CPU path with OpenMP"}


def parity_weibel2d(wl: dict, horizon: int, every: int = 10) -> dict:
    """The 2D FP64 Weibel configuration at full size stepped to its horizon on
    the GPU and in the OpenMP C restatement (exact order: each cell's current
    in particle order, the serial build's result), from the same particles:
    the exact-order current (pic_config.exact_current = 1), compared bit for
    bit at the horizon and in its energies every `every` steps, and the
    default atomic current, whose rounding differences the instability
    amplifies, in its energy curves."""
    import numpy as np

    from oracle import oracle as O
    from pictor_b200 import Particles, PicConfig, Simulation, init_scale

    sc = init_scale(wl["c"], wl["c_ompe"], wl["epc"])
    nx, ny = wl["nx"], wl["ny"]
    g = O.make_grid(2, nx, ny, c=wl["c"], qi=sc["qi"])
    p = O.load_weibel(2, nx, ny, epc=wl["epc"], drift=wl["drift"], temp=wl["temp"], seed=SEED)
    v = p.view()
    host = Particles(*(v[k].copy() for k in ("q", "x", "y", "z", "u", "v", "w")), v["flv"].astype(np.int32))
    o = O.Oracle(g, p.copy(), openmp=True, exact_order=True)
    cap = int(p.used * 1.3) + 65536
    mk = lambda exact: PicConfig(nx=nx, ny=ny, dims=2, c=wl["c"], qi=sc["qi"], precision="fp64",  # noqa: E731
                                 capacity=cap, reorder_period=20, exact_current=exact)
    err = {"exact": {"field": 0.0, "kinetic": 0.0}, "atomic": {"field": 0.0, "kinetic": 0.0}}
    gauss = {"exact": 0.0, "oracle": 0.0}
    t_oracle = t_gpu = 0.0
    with Simulation(mk(1)) as se, Simulation(mk(0)) as sf:
        se.load_particles(host)
        sf.load_particles(host)
        for t in range(1, horizon + 1):
            c0 = time.perf_counter()
            o.step(t, 20)
            c1 = time.perf_counter()
            se.step(1)
            sf.step(1)
            t_oracle += c1 - c0
            t_gpu += time.perf_counter() - c1
            if t % every == 0 or t == horizon:
                ob, oe = o.field_energy()
                of = 0.5 * (ob + oe)
                ok = float(sum(o.particle_energy(sc["masse"])))
                for name, sim in (("exact", se), ("atomic", sf)):
                    d = sim.diagnostics(sc["masse"])
                    fe, ke = 0.5 * (d["B2"] + d["E2"]), float(sum(d["kinetic"]))
                    err[name]["field"] = max(err[name]["field"], abs(fe - of) / of)
                    err[name]["kinetic"] = max(err[name]["kinetic"], abs(ke - ok) / ok)
                    if name == "exact":
                        gauss["exact"] = max(gauss["exact"], d["gauss_linf"] / max(d["rho_max"], 1e-300))
            if t % 100 == 0 or t == horizon:
                res, rmax = o.gauss_residual()
                gauss["oracle"] = max(gauss["oracle"], res / max(rmax, 1e-300))
        gp = se.fetch_particles()
        gf = se.fetch_fields(with_current=False)
        ov = o.p.view()
        same_p = len(gp.x) == o.p.used and all(np.array_equal(getattr(gp, k), ov[k]) for k in ("q", "x", "y", "z", "u", "v", "w", "flv"))
        same_f = all(np.array_equal(getattr(gf, n), getattr(o.f, n)) for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"))
    return {"horizon_steps": horizon, "particles": int(p.used), "energies_every": every,
            "oracle": f"OpenMP C restatement of the reference CPU path, exact order, "
                      f"{os.environ.get('OMP_NUM_THREADS', os.cpu_count())} threads",
            "exact_current": {"bit_exact_particles_at_horizon": bool(same_p),
                              "bit_exact_fields_at_horizon": bool(same_f),
                              "field_energy_rel_diff_max": err["exact"]["field"],
                              "kinetic_energy_rel_diff_max": err["exact"]["kinetic"]},
            "atomic_current": {"field_energy_rel_diff_max": err["atomic"]["field"],
                               "kinetic_energy_rel_diff_max": err["atomic"]["kinetic"]},
            "gauss_linf_over_rho_max": gauss, "seconds": {"oracle": t_oracle, "gpu_both_forms": t_gpu}}


def run_slab_bench(args, ws, rank, local, peak, peak_kind):
    """--workload slab_weibel2d_fp64 / slab_weibel3d_fp32: the 2D FP64 or the
    3D FP32 Weibel grid split along x into one slab per rank
    (pictor_b200.slab; x faces over NCCL, or copied in place on one rank),
    each slab loaded by the device loader (seed + rank); the whole step timed
    with CUDA events, max over ranks."""
    import torch

    from pictor_b200 import init_scale
    from pictor_b200.slab import DistTransport, LocalTransport, Slab, SlabDomain

    wl = WORKLOADS[args.workload]
    sc = init_scale(wl["c"], wl["c_ompe"], wl["epc"])
    dims, prec = wl["dims"], wl["precision"]
    vol = wl["nx"] * wl["ny"] * (wl["nz"] if dims == 3 else 1)
    cap = int(2 * wl["epc"] * vol * 1.04 / ws) + (1 << 16)
    from pictor_b200 import PicConfig

    cfg = PicConfig(nx=wl["nx"], ny=wl["ny"], nz=wl["nz"] if dims == 3 else 1, dims=dims, c=wl["c"], qi=sc["qi"],
                    precision=prec, capacity=cap, reorder_period=20)
    dev = torch.device("cuda", local)
    transport = DistTransport() if ws > 1 else LocalTransport()
    # fixed-size particle boxes (the counts travel on the device, no host
    # wait in a step) of half an x layer of the slab at the configured fill
    box = cap // (wl["nx"] // ws) // 2 + 4096
    dom = SlabDomain([Slab(cfg, rank, ws, dev, out_capacity=box)], transport, queued=True, fixed=True)
    sim = dom.slabs[0].sim
    n_p = sim.init_weibel(wl["epc"], 0.5, wl["drift"], wl["temp"], wl["temp"], SEED + rank)
    sim.reorder()
    dom.step(args.warmup)
    stream = torch.cuda.ExternalStream(sim.stream)
    clocks = ClockSampler(local)
    clocks.start()
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dom.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    ms = max_over_ranks(ws, e0.elapsed_time(e1))
    n_tot = sum_over_ranks(ws, float(n_p))
    d = sim.diagnostics(sc["masse"])
    field = sum_over_ranks(ws, 0.5 * (d["B2"] + d["E2"]))
    dom.close()
    value = n_tot * args.steps / (ms * 1e-3)
    step_bytes = n_tot * bytes_per_particle(dims, prec) + vol * 24 * (8 if prec == "fp64" else 4)
    achieved = step_bytes / (ms / args.steps * 1e-3) / 1e9
    cpu = None if (args.no_cpu or rank != 0) else cpu_sample(WORKLOADS[wl["cpu_workload"]])
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "f32", "data": "synthetic",
            "config": {"workload": args.workload,
                       "global_cells": [wl["nx"], wl["ny"]] + ([wl["nz"]] if dims == 3 else []), "slabs": ws,
                       "slab_cells_x": wl["nx"] // ws, "particles": int(n_tot), "parallelism": f"slab{ws}",
                       "exchange": ("NCCL point-to-point between ranks" if ws > 1 else "x faces copied on the rank")
                       + ", ordered on the library's stream; particles in fixed-size boxes of "
                       + f"{box} (their counts on the device): no host wait in a step",
                       "l2": ("particles and fields smaller than L2 at this size" if dims == 2 else
                              "inputs larger than L2 (particle state >> 126 MB)")},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "kernel": "whole slab step (phases and host-driven exchanges)",
                         "peak_kind": peak_kind},
            "cpu_baseline": cpu, "e2e": None, "gpu_launches": None, "clocks": clk,
            "energy": {"field": field},
        }
        print(json.dumps(line))
    return 0


def run_ensemble_bench(args, ws, rank, local, peak, peak_kind):
    """--workload ensemble64: this rank's share of the 64 runs (largest-first
    plan), stepped together with pic_step_many after the per-size-class
    autotuner, against the same runs in the plain FP64 form one at a time."""
    import torch

    from pictor_b200.ensemble import ensemble_runs, partition, run_batched, tune_classes

    wl = WORKLOADS[args.workload]
    runs = ensemble_runs(wl["runs"], steps=args.steps)
    mine = [runs[i] for i in partition(runs, ws)[rank]]
    t0 = time.perf_counter()
    tunings = tune_classes(mine)
    tune_s = time.perf_counter() - t0
    horizon = args.horizon if args.horizon is not None else wl.get("horizon", 0)
    if args.no_fp64:
        horizon = 0
    run_batched(mine, args.warmup, "fp32", tunings)                      # warm-up (graph capture, clocks)
    clocks = ClockSampler(local)
    clocks.start()
    barrier(ws)
    res32, t32 = run_batched(mine, args.steps, "fp32", tunings, horizon=horizon)
    barrier(ws)
    clk = clocks.stop()
    secs = max_over_ranks(ws, t32["seconds"])
    ps = sum_over_ranks(ws, t32["particle_steps"])
    value = ps / secs
    # the same runs with one launch per phase for each group of runs (pic_step_batched)
    run_batched(mine, args.warmup, "fp32", tunings, per_phase=True)          # warm-up
    barrier(ws)
    resp, tp = run_batched(mine, args.steps, "fp32", tunings, per_phase=True)
    secs_p = max_over_ranks(ws, tp["seconds"])
    per_phase = {"value": sum_over_ranks(ws, tp["particle_steps"]) / secs_p, "seconds": secs_p,
                 "gpu_launches": tp["launches"],
                 "max_kinetic_rel_diff_vs_streams": max(abs(sum(a["kinetic"]) - sum(b["kinetic"])) / abs(sum(b["kinetic"]))
                                                        for a, b in zip(resp, res32)),
                 "form": "pic_step_batched: the runs in 4 groups, each phase of a group one launch over all "
                         "its runs, one CUDA graph per group and step"}
    # and as one persistent launch per span between reorders (pic_step_persistent)
    run_batched(mine, args.warmup, "fp32", tunings, persistent=True)         # warm-up
    barrier(ws)
    resq, tq = run_batched(mine, args.steps, "fp32", tunings, persistent=True)
    secs_q = max_over_ranks(ws, tq["seconds"])
    persistent = {"value": sum_over_ranks(ws, tq["particle_steps"]) / secs_q, "seconds": secs_q,
                  "gpu_launches": tq["launches"],
                  "max_kinetic_rel_diff_vs_streams": max(abs(sum(a["kinetic"]) - sum(b["kinetic"])) / abs(sum(b["kinetic"]))
                                                         for a, b in zip(resq, res32)),
                  "form": "pic_step_persistent: every phase of every run in one launch of 3 CTAs per SM per "
                          "span of steps between reorders, work items ordered by per-run counters"}
    fp64 = None
    if not args.no_fp64:
        def errs(r32, r64):
            ef = max(abs((a["B2"] + a["E2"]) - (b["B2"] + b["E2"])) / max(b["B2"] + b["E2"], 1e-300)
                     for a, b in zip(r32, r64))
            et = max(abs((0.5 * (a["B2"] + a["E2"]) + sum(a["kinetic"])) - (0.5 * (b["B2"] + b["E2"]) + sum(b["kinetic"])))
                     / abs(0.5 * (b["B2"] + b["E2"]) + sum(b["kinetic"])) for a, b in zip(r32, r64))
            return ef, et
        # the same runs in the plain FP64 form, stepped together as the FP32 runs are (pic_step_many)
        res64, t64 = run_batched(mine, args.steps, "fp64", None, batched=True, horizon=horizon)
        secs64 = max_over_ranks(ws, t64["seconds"])
        v64 = sum_over_ranks(ws, t64["particle_steps"]) / secs64
        err_f, err_t = errs(res32, res64)
        # and one after the other
        _, t64s = run_batched(mine, args.steps, "fp64", None, batched=False)
        secs64s = max_over_ranks(ws, t64s["seconds"])
        v64s = sum_over_ranks(ws, t64s["particle_steps"]) / secs64s
        fp64 = {"value": v64, "seconds": secs64, "speedup_fp32_batched_over_fp64": value / v64,
                "max_field_energy_rel_err": err_f, "max_total_energy_rel_err": err_t,
                "errors_at": f"step {args.steps}",
                "form": "plain FP64 reference layout, the runs stepped together on their own streams (pic_step_many)",
                "one_after_the_other": {"value": v64s, "seconds": secs64s,
                                        "speedup_fp32_batched_over_fp64": value / v64s}}
        if horizon and "horizon" in t32 and "horizon" in t64:
            hf, ht = errs(t32["horizon"], t64["horizon"])
            fp64["horizon"] = {"steps": horizon, "max_field_energy_rel_err": hf, "max_total_energy_rel_err": ht,
                               "form": "every run continued to step 500 in both forms; the largest per-run "
                                       "relative difference"}
    # end to end: particles from pinned FP64 host arrays for every run, the steps, the diagnostics
    from pictor_b200.ensemble import make_run, size_class
    from pictor_b200.simulation import step_many

    sims, hosts = [], []
    for spec in mine:
        sim, sc = make_run(spec, "fp32", tunings.get(size_class(spec)))
        p = sim.fetch_particles()
        hosts.append(type(p)(*(torch.from_numpy(getattr(p, k)).pin_memory().numpy()
                               for k in ("q", "x", "y", "z", "u", "v", "w", "flv"))))
        sims.append((sim, sc))
    h2d = sum(len(h.x) for h in hosts) * (7 * 8 + 4)
    barrier(ws)
    torch.cuda.synchronize()
    te = time.perf_counter()
    for (sim, _), hp in zip(sims, hosts):
        sim.load_particles(hp)
        sim.reorder()
    step_many([s for s, _ in sims], args.steps)
    for sim, sc in sims:
        sim.diagnostics(sc["masse"])
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(ws, time.perf_counter() - te)
    for sim, _ in sims:
        sim.close()
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        from oracle import oracle as O

        O.build()
        cpu = cpu_sample(wl)
    n_bytes = sum(2 * r.ppc * r.nx * r.ny * bytes_per_particle(2, "fp32") + r.nx * r.ny * bytes_per_cell_mover("fp32")
                  for r in mine)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "ensemble64", "runs": wl["runs"], "runs_this_rank": len(mine),
                       "grids": "64^2..512^2", "ppc_per_species": "4..32", "seed": "2930 + run",
                       "parallelism": f"ensemble shards over {ws} rank(s)", "autotune_seconds": tune_s,
                       "tunings": {f"{k[0]}x{k[1]}/ppc{k[2]}": {"brick": list(v.brick[:2]),
                                                                 "reorder_period": v.reorder_period}
                                   for k, v in tunings.items()},
                       "l2": "run state of the rank (GBs) larger than L2"},
            "roofline": {"bound": "hbm", "achieved": n_bytes * args.steps / t32["seconds"] / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": n_bytes * args.steps / t32["seconds"] / 1e9 / peak,
                         "traffic": None, "kernel": "batched step (k_move_f32_tiled<2> dominant), aggregate",
                         "peak_kind": peak_kind},
            "gpu_launches": t32["launches"],
            "clocks": clk,
            "e2e": {"value": ps / e2e_s, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d / args.steps,
                    "d2h_bytes_per_step": 8 * 6 * len(mine) / args.steps, "seconds": e2e_s,
                    "includes": "pic_load_particles of every run from pinned FP64 host arrays + reorder + "
                                "pic_step_many + pic_diagnostics"},
        }
        line["one_launch_per_phase"] = per_phase
        line["persistent"] = persistent
        if fp64:
            line["fp64"] = fp64
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_adjoint_bench(args, rank, local, peak, peak_kind):
    """--workload adjoint128: the gradient of the time-integrated magnetic
    energy (forward with checkpoints + reverse sweep) in the FP32 form, the
    FP64 reference adjoint on the same run, and central finite differences of
    the FP64 forward (h = 1e-4 of each parameter / a unit momentum direction)."""
    import numpy as np
    import torch

    from pictor_b200 import PicConfig, init_scale
    from pictor_b200.adjoint import Adjoint

    wl = WORKLOADS[args.workload]
    steps, K = wl["nsteps"], wl["checkpoint"]
    sc = init_scale(wl["c"], wl["c_ompe"], wl["epc"])
    n_cells = wl["nx"] * wl["ny"]
    cap = int(2 * wl["epc"] * n_cells * 1.2) + 4096
    load = (wl["epc"], 0.5, wl["drift"], wl["temp"], wl["temp"], SEED)

    def make(prec):
        return Adjoint(PicConfig(nx=wl["nx"], ny=wl["ny"], dims=2, c=wl["c"], qi=sc["qi"], precision=prec,
                                 capacity=cap, reorder_period=0))

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0

    out = {}
    for prec in ("fp32", "fp64"):
        with make(prec) as a:
            n = a.init_weibel(*load)
            for _ in range(max(1, args.warmup // 3)):        # warm-up: allocations, graph capture, clocks
                a.forward(steps, K)
                a.gradient()
            clocks = ClockSampler(local)
            clocks.start()
            J, tf = timed(lambda: a.forward(steps, K))
            g, tg = timed(lambda: a.gradient())
            clk = clocks.stop()
            out[prec] = {"n": n, "J": J, "t_forward": tf, "t_gradient": tg, "g": g, "clocks": clk}
    g32, g64 = out["fp32"]["g"], out["fp64"]["g"]
    v32 = np.concatenate([g32[k] for k in ("u", "v", "w")])
    v64 = np.concatenate([g64[k] for k in ("u", "v", "w")])
    # agreement with central differences of the FP64 forward (h = 1e-4 of each
    # parameter, unit momentum direction), and of the FP32 with the FP64
    # gradient, as a function of the horizon: the Weibel run is unstable, so
    # gradients grow exponentially with the horizon and the zigzag current's
    # jumps make long-horizon finite differences meaningless
    sweep = []
    if not args.no_sweep:
        with make("fp64") as a64, make("fp32") as a32:
            a64.init_weibel(*load)
            a32.init_weibel(*load)
            p0, sgn = a64.fetch_particles()
            rng = np.random.default_rng(SEED)
            d = rng.normal(size=(3, len(p0.x)))
            d /= np.sqrt((d * d).sum())

            def fd(fn, h):
                return (fn(h) - fn(-h)) / (2 * h)

            for H in (10, 25, 50, 100, 200, 400):
                if H > steps:
                    break
                KH = min(K, H)
                a64.init_weibel(*load)
                a64.branches("record")
                a64.forward(H, KH)
                g = a64.gradient()
                a32.forward(H, KH)
                gs = a32.gradient()

                def j_load(dd, dti):
                    a64.init_weibel(wl["epc"], 0.5, wl["drift"] + dd, wl["temp"] + dti, wl["temp"], SEED)
                    return a64.forward(H, KH)

                def j_dir(h):
                    p = type(p0)(*(getattr(p0, f).copy() for f in p0.NAMES))
                    p.u += h * d[0]
                    p.v += h * d[1]
                    p.w += h * d[2]
                    a64.load_particles(p, sgn)
                    return a64.forward(H, KH)

                def fd_checks():
                    return [("drift", g["drift"], fd(lambda h: j_load(h, 0), 1e-4 * wl["drift"])),
                            ("temp_ion", g["temp_ion"], fd(lambda h: j_load(0, h), 1e-4 * wl["temp"])),
                            ("momenta_dir", float((g["u"] * d[0] + g["v"] * d[1] + g["w"] * d[2]).sum()),
                             fd(j_dir, 1e-4))]

                # perturbed runs replaying the base run's discrete decisions (smooth in the inputs),
                # then free ones (straddling the zigzag current's jumps)
                a64.branches("replay")
                frozen = fd_checks()
                a64.branches("free")
                checks = fd_checks()
                v64h = np.concatenate([g[k] for k in ("u", "v", "w")])
                v32h = np.concatenate([gs[k] for k in ("u", "v", "w")])
                sweep.append({"steps": H, "grad_norm_momenta": float(np.linalg.norm(v64h)),
                              "fp32_vs_fp64_rel_l2": float(np.linalg.norm(v32h - v64h) / np.linalg.norm(v64h)),
                              "fd": [{"param": nme, "adjoint": ad, "fd": f, "rel_err": abs(ad - f) / max(abs(f), 1e-300)}
                                     for nme, ad, f in checks],
                              "fd_frozen_branches": [{"param": nme, "adjoint": ad, "fd": f,
                                                      "rel_err": abs(ad - f) / max(abs(f), 1e-300)}
                                                     for nme, ad, f in frozen]})
    agree = [r["steps"] for r in sweep if all(c["rel_err"] <= 1e-2 for c in r["fd"])]
    agree_frozen = [r["steps"] for r in sweep if all(c["rel_err"] <= 1e-3 for c in r["fd_frozen_branches"])]
    fdc = sweep[-1]["fd"] if sweep else []
    n = out["fp32"]["n"]
    t32 = out["fp32"]["t_forward"] + out["fp32"]["t_gradient"]
    t64 = out["fp64"]["t_forward"] + out["fp64"]["t_gradient"]
    value = n * steps / t32
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": 1, "steps": steps,
            "warmup": args.warmup, "ms_per_step": t32 / steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "adjoint128", "cells": [wl["nx"], wl["ny"]], "particles": n,
                       "particles_per_cell_per_species": wl["epc"], "drift_c": wl["drift"],
                       "thermal_c": math.sqrt(wl["temp"] / 2), "courant": wl["c"], "steps": steps,
                       "checkpoint_every": K, "objective": "sum_t 1/2 sum_cells |B_t|^2",
                       "counted": "particle-steps of the run per second of forward + reverse sweep",
                       "l2": "tape of one segment (GBs at this size) larger than L2"},
            "objective": {"fp32": out["fp32"]["J"], "fp64": out["fp64"]["J"]},
            "timing_s": {"fp32_forward": out["fp32"]["t_forward"], "fp32_gradient": out["fp32"]["t_gradient"],
                         "fp64_forward": out["fp64"]["t_forward"], "fp64_gradient": out["fp64"]["t_gradient"]},
            "fp64": {"value": n * steps / t64, "speedup_fp32_over_fp64": t64 / t32,
                     "momentum_gradient_rel_l2_fp32_vs_fp64": float(np.linalg.norm(v32 - v64) / np.linalg.norm(v64)),
                     "drift_gradient": {"fp32": g32["drift"], "fp64": g64["drift"]},
                     "temp_gradient": {"fp32": [g32["temp_ion"], g32["temp_elc"]],
                                       "fp64": [g64["temp_ion"], g64["temp_elc"]]}},
            "fd_checks_fp64_full_horizon": fdc,
            "fd_mismatch_fraction_full_horizon": (sum(1 for c in fdc if c["rel_err"] > 1e-2) / len(fdc)) if fdc else None,
            "horizon_sweep": sweep,
            "fd_agreement_1e-2_up_to_steps": max(agree) if agree else 0,
            "fd_frozen_branches_agreement_1e-3_up_to_steps": max(agree_frozen) if agree_frozen else 0,
            "roofline": {"bound": "hbm", "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
                         "traffic": None, "kernel": "k_move_T (mover adjoint), latency/atomic bound at this size",
                         "peak_kind": peak_kind},
            # forward: 2 B half steps, mover, E update, energy per step; gradient: the 4 kernels of each
            # recomputed step, the 7 of each reverse step, the parameter reduction and 5 conversions
            "gpu_launches": 5 * steps + 12 * steps + 6,
            "clocks": out["fp32"]["clocks"],
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 3 * 8 * n / steps,
                    "includes": "device loader, forward, reverse sweep, gradient copied to host"},
        }
        print(json.dumps(line), flush=True)
    return 0


def cpu_sample_cyl(wl: dict, target_s: float = 12.0):
    """The cylindrical CPU step (C restatement of cyl_movdep_strang.F90 +
    cyl_em_update*.F90) on a 64 x 8 x 128 sub-box with the same plasma."""
    from oracle import oracle as O

    qi = O.init_scale(wl["c"], wl["c_ompe"], wl["epc"])[0]
    g = O.make_grid(3, 64, wl["ny"], 128, c=wl["c"], qi=qi, fdtd="lehe", qm=(1.0, -1.0))
    # the loader's per-component spread is sqrt(temp / 2)
    temp = 2.0 * (wl["thermal"] * wl["c"]) ** 2
    p = O.cyl_load_uniform(g, 2, 2, 2, 1.0, temp, -1.0, 2, SEED, 64 * wl["ny"] * 128 * 8 * 2)
    o = O.CylOracle(g, p)
    o.step(1)
    n_steps, t0, t = 0, time.perf_counter(), 1
    while True:
        t += 1
        o.step(t)
        n_steps += 1
        el = time.perf_counter() - t0
        if el >= target_s or n_steps >= 200:
            break
    return {"value": p.used * n_steps / el, "unit": "particle-steps/s", "cores": 1, "kind": "port",
            "sample": f"64x{wl['ny']}x128 cells, {p.used} particles, {n_steps} steps (same plasma, no bunch), FP64, "
                      "C restatement of the reference cylindrical CPU path, serial"}


def run_cyl_bench(args, rank, local, peak, peak_kind):
    """--workload cyl_wake: the cylindrical wakefield run in the reference's
    theta-gridded FP64 form (the form this library has for cylindrical
    geometry), particles from pictor_b200.setups.cyl_wakefield."""
    import torch

    from pictor_b200 import Particles, PicConfig, Simulation, init_scale
    from pictor_b200.setups import cyl_wakefield

    wl = WORKLOADS[args.workload]
    sc = init_scale(wl["c"], wl["c_ompe"], wl["epc"])
    p, info = cyl_wakefield(wl["nx"], wl["nz"], wl["ny"], wl["c"], thermal=wl["thermal"], bunch_gamma=wl["bunch_gamma"],
                            bunch_peak=wl["bunch_peak"], bunch_sigma_r=wl["bunch_sigma_r"],
                            bunch_sigma_z=wl["bunch_sigma_z"], seed=SEED)
    n_p = len(p.x)
    cfg = PicConfig(nx=wl["nx"], ny=wl["ny"], nz=wl["nz"], dims=3, c=wl["c"], qi=sc["qi"], qm=(1.0, -1.0),
                    fdtd="lehe", geom="cylindrical", precision=wl["precision"], capacity=2 * n_p + 4096,
                    reorder_period=20, rmin=-0.5, inc_axis=1, cyl_modes=wl.get("cyl_modes", 0))
    pinned = Particles(*(torch.from_numpy(getattr(p, k)).pin_memory().numpy() for k in Particles.NAMES))
    with Simulation(cfg) as sim:
        sim.load_particles(pinned)
        sim.reorder()
        sim.step(args.warmup)
        clocks = ClockSampler(local)
        clocks.start()
        ms, phases, launches = timed_steps(sim, args.steps, 1, profile=True)
        clk = clocks.stop()
        d = sim.diagnostics(sc["masse"])
        # end to end: the particles from pinned host memory, the steps, diagnostics, the fields back
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.load_particles(pinned)
        sim.reorder()
        sim.step(args.steps)
        sim.diagnostics(sc["masse"])
        f = sim.fetch_fields(with_current=False)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
    value = n_p * args.steps / (ms * 1e-3)
    move_ms = phases["ms"]["move"] / max(phases["steps"], 1)
    n_cells = wl["nx"] * wl["ny"] * wl["nz"]
    bytes_move = n_p * bytes_per_particle(3, wl["precision"]) + n_cells * bytes_per_cell_mover(wl["precision"])
    # the FP32 form against the FP64 form of the same run to the configuration's horizon
    horizon_cmp = None
    horizon = args.horizon if args.horizon is not None else wl.get("horizon", 0)
    if wl["precision"] == "fp32" and horizon and not args.no_fp64:
        curves = {}
        for prec in ("fp32", "fp64"):
            with Simulation(dataclasses.replace(cfg, precision=prec)) as sim:
                sim.load_particles(pinned)
                sim.reorder()
                curves[prec] = energy_curve(sim, sc, 0, horizon, every=100)
        horizon_cmp = {"steps": horizon, "every": 100, **curve_errors(curves["fp32"], curves["fp64"]),
                       "form": "the FP32 form and the FP64 form of the same run (same field solve), "
                               "energies compared every 100 steps"}
    cpu = None if args.no_cpu else cpu_sample_cyl(wl)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if wl["precision"] == "fp32" else "f64", "data": "synthetic",
            "config": {"workload": args.workload,
                       "form": (("field solve on azimuthal modes m=0,1, particles on the theta grid, "
                                 + ("FP32 (cell-relative particles)" if wl["precision"] == "fp32" else "FP64"))
                                if wl.get("cyl_modes", 0) else
                                "FP32 cell-relative particles, theta-gridded FP32 fields" if wl["precision"] == "fp32"
                                else "theta-gridded FP64 (the reference's representation)"),
                       "cells_r_theta_z": [wl["nx"], wl["ny"], wl["nz"]], "particles": n_p, **info,
                       "courant": wl["c"], "c_ompe": wl["c_ompe"], "fdtd": "lehe (z)", "reorder_period": 20,
                       "l2": "particle state (GBs) larger than L2"},
            "roofline": {"bound": "hbm", "achieved": bytes_move / (move_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": bytes_move / (move_ms * 1e-3) / 1e9 / peak, "traffic": None,
                         "kernel": "k_cyl_move_f32_tiled" if wl["precision"] == "fp32" else "k_cyl_move",
                         "launch_ms": move_ms, "peak_kind": peak_kind},
            "phases_ms_per_step": {k: v / max(phases["steps"], 1) for k, v in phases["ms"].items()},
            "gpu_launches": launches, "clocks": clk,
            "energy": {"field": 0.5 * (d["B2"] + d["E2"]), "kinetic": float(sum(d["kinetic"]))},
            **({"fp32_vs_fp64": horizon_cmp} if horizon_cmp else {}),
            "e2e": {"value": n_p * args.steps / e2e_s, "unit": "particle-steps/s",
                    "h2d_bytes_per_step": n_p * 60 / args.steps,
                    "d2h_bytes_per_step": 6 * 8 * (wl["nx"] + 5) * (wl["ny"] + 5) * (wl["nz"] + 5) / args.steps,
                    "seconds": e2e_s},
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    return 0


def run_reference(args):
    """--impl reference: the reference's CPU algorithm (C restatement of the
    Fortran CPU path; the Fortran build is not available here) on the host."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = WORKLOADS[args.workload]
    from oracle import oracle as O

    O.build()
    target = max(5.0, min(60.0, 3.0 * args.steps))
    base = cpu_sample_cyl(wl, target_s=target) if args.workload.startswith("cyl") else cpu_sample(wl, target_s=target)
    line = {
        "metric": METRIC, "value": base["value"], "unit": "particle-steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": args.workload, **{k: v for k, v in wl.items()}, "seed": SEED},
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="weibel3d_fp32")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffers) run")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-sweep", action="store_true", help="adjoint128: skip the finite-difference horizon sweep")
    ap.add_argument("--parity", action="store_true",
                    help="weibel2d_fp64: step the full configuration to its horizon on the GPU and in the "
                         "OpenMP C restatement and report the differences")
    ap.add_argument("--horizon", type=int, default=None,
                    help="steps to which the FP32 and FP64 runs are continued for the energy comparison "
                         "(default: the configuration's; 0 = none)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import numpy as np
    import torch

    from pictor_b200 import build

    build.build()
    ws, rank, local = dist_setup(args.gpus)
    if args.workload == "ensemble64":
        peak, peak_kind = measured_peaks()
        return run_ensemble_bench(args, ws, rank, local, peak, peak_kind)
    if args.workload == "adjoint128":
        peak, peak_kind = measured_peaks()
        return run_adjoint_bench(args, rank, local, peak, peak_kind)
    if args.workload.startswith("slab_"):
        peak, peak_kind = measured_peaks()
        return run_slab_bench(args, ws, rank, local, peak, peak_kind)
    if args.workload.startswith("cyl_wake"):
        peak, peak_kind = measured_peaks()
        return run_cyl_bench(args, rank, local, peak, peak_kind)
    wl = WORKLOADS[args.workload]
    prec = wl["precision"]
    seed = SEED + rank
    peak, peak_kind = measured_peaks()

    # ---- headline: the workload in its own precision, inputs resident -----
    sim, sc = make_sim(wl, prec)
    n_p = sim.init_weibel(wl["epc"], 0.5, wl["drift"], wl["temp"], wl["temp"], seed)
    sim.reorder()                      # ReorderPrtl at Startups (MAIN.F90:307)
    sim.step(args.warmup)
    clocks = ClockSampler(local)
    clocks.start()
    ms, phases, launches = timed_steps(sim, args.steps, ws, profile=True)
    clk = clocks.stop()
    e32 = energies(sim, sc)
    # the run continued to the configuration's horizon, energies every 20 steps
    horizon = args.horizon if args.horizon is not None else wl.get("horizon", 0)
    done = args.warmup + args.steps
    curve32 = {done: e32}
    if not args.no_fp64 and prec == "fp32" and horizon > done:
        curve32.update(energy_curve(sim, sc, done, horizon))
    ms_max = max_over_ranks(ws, ms)
    n_tot = sum_over_ranks(ws, float(n_p))
    value = n_tot * args.steps / (ms_max * 1e-3)

    n_cells = wl["nx"] * wl["ny"] * (wl["nz"] if wl["dims"] == 3 else 1)
    move_ms = phases["ms"]["move"] / max(phases["steps"], 1)
    bytes_move = n_p * bytes_per_particle(wl["dims"], prec) + n_cells * bytes_per_cell_mover(prec)
    achieved = bytes_move / (move_ms * 1e-3) / 1e9
    step_bytes = (n_p * bytes_per_particle(wl["dims"], prec) + n_cells * 24 * (4 if prec == "fp32" else 8))
    sim.close()
    del sim

    # ---- FP64 reference form on the same seed -------------------------------
    fp64 = None
    if not args.no_fp64 and prec == "fp32":
        sim64, _ = make_sim(wl, "fp64")
        sim64.init_weibel(wl["epc"], 0.5, wl["drift"], wl["temp"], wl["temp"], seed)
        sim64.reorder()
        sim64.step(args.warmup)
        ms64, ph64, _ = timed_steps(sim64, args.steps, ws, profile=True)
        e64 = energies(sim64, sc)
        curve64 = {done: e64}
        if horizon > done:
            curve64.update(energy_curve(sim64, sc, done, horizon))
        ms64 = max_over_ranks(ws, ms64)
        v64 = n_tot * args.steps / (ms64 * 1e-3)
        fp64 = {"value": v64, "ms_per_step": ms64 / args.steps, "speedup_fp32_over_fp64": value / v64,
                "field_energy_rel_err": abs(e32["field"] - e64["field"]) / max(abs(e64["field"]), 1e-300),
                "total_energy_rel_err": abs((e32["field"] + e32["kinetic"]) - (e64["field"] + e64["kinetic"]))
                / max(abs(e64["field"] + e64["kinetic"]), 1e-300),
                "field_energy_fp64": e64["field"], "field_energy_fp32": e32["field"],
                "gauss_linf_over_rho": e64["gauss_linf"] / max(e64["rho_max"], 1e-300),
                "move_ms": ph64["ms"]["move"] / max(ph64["steps"], 1),
                "errors_at": f"step {done} (the first three keys above)"}
        if horizon > done:
            fp64["horizon"] = {"steps": horizon, "every": 20, **curve_errors(curve32, curve64),
                               "form": "both runs from the same seed to the configuration's horizon, energies "
                                       "compared every 20 steps"}
        sim64.close()
        del sim64

    # ---- end to end through the C ABI with host buffers ---------------------
    e2e = None
    if not args.no_e2e:
        sim, sc = make_sim(wl, prec)
        sim.init_weibel(wl["epc"], 0.5, wl["drift"], wl["temp"], wl["temp"], seed)
        host = sim.fetch_particles()  # reference-layout FP64 host arrays
        pinned = {}
        for k in ("q", "x", "y", "z", "u", "v", "w", "flv"):
            a = getattr(host, k)
            t = torch.from_numpy(a).pin_memory()
            pinned[k] = t
        del host
        from pictor_b200 import Particles

        hp = Particles(*(pinned[k].numpy() for k in ("q", "x", "y", "z", "u", "v", "w", "flv")))
        # the result's host arrays, pinned like the inputs
        from pictor_b200 import Fields

        shape = tuple(sim.cfg.shape)
        out_bufs = [torch.empty(int(np.prod(shape)), dtype=torch.float64).pin_memory() for _ in range(6)]
        fout = Fields(*(t.numpy().reshape(shape, order="F") for t in out_bufs))
        stream = torch.cuda.ExternalStream(sim.stream)
        sim.load_particles(hp)
        sim.reorder()
        sim.step(args.warmup)
        barrier(ws)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.load_particles(hp)                 # host -> device: the run's particle state
        sim.reorder()                          # ReorderPrtl at Startups
        sim.step(args.steps)
        d = sim.diagnostics(sc["masse"])       # device -> host: energies, Gauss residual
        f = sim.fetch_fields(with_current=False, out=fout)  # device -> host: the fields
        e1.record(stream)
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) * 1e3
        barrier(ws)
        ms_e2e = max_over_ranks(ws, max(wall, e0.elapsed_time(e1)))
        h2d = n_p * (7 * 8 + 4)
        d2h = 6 * (wl["nx"] + 5) * (wl["ny"] + 5) * ((wl["nz"] + 5) if wl["dims"] == 3 else 1) * 8 + 8 * len(d["kinetic"]) + 32
        e2e = {"value": n_tot * args.steps / (ms_e2e * 1e-3), "unit": "particle-steps/s",
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "ms": ms_e2e, "includes": "pic_load_particles from pinned FP64 host arrays + K steps + "
                                          "pic_diagnostics + pic_fetch_fields into pinned FP64 host arrays"}
        sim.close()
        del sim, f

    # ---- CPU baseline (rank 0, N=1) -----------------------------------------
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        from oracle import oracle as O

        O.build()
        cpu = cpu_sample(wl)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if prec == "fp32" else "f64", "data": "synthetic",
            "config": {"workload": args.workload, "cells": [wl["nx"], wl["ny"], wl["nz"]][: wl["dims"]],
                       "particles_per_gpu": n_p, "particles_per_cell_per_species": wl["epc"],
                       "drift_c": wl["drift"], "thermal_c": math.sqrt(wl["temp"] / 2), "courant": wl["c"],
                       "c_ompe": wl["c_ompe"], "reorder_period": 20, "seed": SEED, "parallelism": f"replicas{ws}",
                       "l2": "inputs larger than L2 (particle state >> 126 MB)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic_per_launch(wl, n_p), "traffic_source": TRAFFIC_SOURCE,
                         "kernel": mover_kernel(wl, prec),
                         "algorithmic_bytes_per_launch": bytes_move, "launch_ms": move_ms,
                         "peak_kind": peak_kind, "step_algorithmic_GBs": step_bytes / (ms_max / args.steps * 1e-3) / 1e9},
            "phases_ms_per_step": {k: v / max(phases["steps"], 1) for k, v in phases["ms"].items()},
            "gpu_launches": launches,
            "clocks": clk,
            "energy": {k: e32[k] for k in ("field", "kinetic", "gauss_linf", "rho_max")},
        }
        if fp64:
            line["fp64"] = fp64
        if e2e:
            line["e2e"] = e2e
        if cpu:
            line["cpu_baseline"] = cpu
        if args.parity and args.workload == "weibel2d_fp64" and ws == 1:
            line["parity"] = parity_weibel2d(wl, args.horizon or wl["horizon"])
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
