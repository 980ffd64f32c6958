"""Multi-rank path of the ensemble form on CPU: world_size-2 gloo process
groups check that every rank derives the same plan, that the plan covers
every run exactly once with balanced load, and that the final gather returns
all results on every rank.  The per-run stepping is replaced by a host stub
(no GPU here); the stub records which rank ran which run."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from pictor_b200.ensemble import ensemble_runs, imbalance, partition


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from pictor_b200.ensemble import ensemble_runs, run_ensemble

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    runs = ensemble_runs(16, steps=10)

    def stub(spec):
        return {"run": spec.run, "rank": rank, "particles": spec.particles}

    res = run_ensemble(runs, rank, world, runner=stub)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, res))


def test_partition_covers_every_run_once_and_balances():
    runs = ensemble_runs(64, steps=500)
    for ws in (1, 2, 4, 8):
        plan = partition(runs, ws)
        flat = sorted(i for p in plan for i in p)
        assert flat == list(range(64))
        if ws <= 4:
            assert imbalance(runs, plan) < 1.2
    assert partition(runs, 4) == partition(runs, 4)


def test_ensemble_draw_is_seeded_per_run():
    a, b = ensemble_runs(8), ensemble_runs(8)
    assert [r.nx for r in a] == [r.nx for r in b]
    assert all(r.seed == 2930 + r.run for r in a)
    assert all(r.nx in (64, 128, 256, 512) and r.ppc in (4, 8, 16, 32) for r in a)
    assert all(0.1 <= r.drift <= 0.9 and 0.01 <= r.sigma <= 0.1 for r in a)


def test_two_rank_gloo_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0] == out[1]                      # every rank holds every result
    assert [d["run"] for d in out[0]] == list(range(16))
    plan = partition(ensemble_runs(16, steps=10), 2)
    for d in out[0]:
        assert d["run"] in plan[d["rank"]]       # each run stepped by its planned rank only
