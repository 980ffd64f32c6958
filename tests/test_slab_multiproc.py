"""Host side of the slab decomposition along x on CPU: the ring transport
between gloo ranks (2 and 3 ranks: each rank's from_left is its left
neighbour's to_right, also when both neighbours are the same rank), the
variable-size particle exchange (counts first, nothing sent for a zero
count), and the split of a global state into slabs and back."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pictor_b200 import Fields, Particles
from pictor_b200.slab import (LocalTransport, exchange_particle_buffers, join_interior, join_particles,
                              slab_width, split_fields, split_particles)


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    from pictor_b200.slab import DistTransport, exchange_particle_buffers

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    t = DistTransport()
    # fixed-size face buffers
    tl, tr = torch.full((6,), 10.0 * rank + 1), torch.full((6,), 10.0 * rank + 2)
    fl, fr = torch.zeros(6), torch.zeros(6)
    t.exchange([(tl, tr)], [(fl, fr)])
    # variable-size particle buffers: rank r sends r particles left and
    # (r + 1) % 2 right, 8 words each, tagged by sender and direction
    nl, nr = rank, (rank + 1) % 2
    out_l = torch.full((8 * nl,), 100.0 * rank + 1)
    out_r = torch.full((8 * nr,), 100.0 * rank + 2)
    got = exchange_particle_buffers(t, [(out_l, out_r)], [(nl, nr)], lambda n: torch.empty(8 * n))
    (bl, cl), (br, cr) = got[0]
    res = {"fl": fl.tolist(), "fr": fr.tolist(), "cl": cl, "cr": cr,
           "bl": None if bl is None else bl.tolist(), "br": None if br is None else br.tolist()}
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, res))


@pytest.mark.parametrize("world", [2, 3])
def test_ring_transport_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        left, right = (r - 1) % world, (r + 1) % world
        assert out[r]["fl"] == [10.0 * left + 2] * 6          # the left neighbour's to_right
        assert out[r]["fr"] == [10.0 * right + 1] * 6         # the right neighbour's to_left
        n_from_left, n_from_right = (left + 1) % 2, right     # their right- / left-bound counts
        assert (out[r]["cl"], out[r]["cr"]) == (n_from_left, n_from_right)
        assert out[r]["bl"] == ([100.0 * left + 2] * (8 * n_from_left) if n_from_left else None)
        assert out[r]["br"] == ([100.0 * right + 1] * (8 * n_from_right) if n_from_right else None)


def test_local_transport_ring_matches_distributed_pairing():
    import torch

    n = 3
    sends = [(torch.full((2,), 10.0 * s + 1), torch.full((2,), 10.0 * s + 2)) for s in range(n)]
    recvs = [(torch.zeros(2), torch.zeros(2)) for _ in range(n)]
    LocalTransport().exchange(sends, recvs)
    for s in range(n):
        assert recvs[s][0].tolist() == [10.0 * ((s - 1) % n) + 2] * 2
        assert recvs[s][1].tolist() == [10.0 * ((s + 1) % n) + 1] * 2
    counts = [(s, 2 * s) for s in range(n)]
    outs = [(torch.full((8 * s,), float(s)), torch.full((16 * s,), float(-s))) for s in range(n)]
    got = exchange_particle_buffers(LocalTransport(), outs, counts, lambda k: torch.empty(8 * k))
    for s in range(n):
        (bl, cl), (br, cr) = got[s]
        assert cl == 2 * ((s - 1) % n) and cr == (s + 1) % n
        assert (bl is None) == (cl == 0) and (br is None) == (cr == 0)
        if cl:
            assert bl.tolist() == [float(-((s - 1) % n))] * (8 * cl)
        if cr:
            assert br.tolist() == [float((s + 1) % n)] * (8 * cr)


def test_split_and_join():
    rng = np.random.default_rng(4)
    nx, ny, nz, S = 24, 6, 6, 3
    w = slab_width(nx, S)
    assert w == 8
    with pytest.raises(ValueError):
        slab_width(24, 5)
    n = 500
    p = Particles(rng.normal(size=n), rng.uniform(3, nx + 3, n), rng.uniform(3, ny + 3, n), rng.uniform(3, nz + 3, n),
                  rng.normal(size=n), rng.normal(size=n), rng.normal(size=n), rng.integers(1, 3, n).astype(np.int32))
    parts = split_particles(p, nx, S)
    assert sum(len(q) for q in parts) == n
    for q in parts:
        assert ((q.x >= 3.0) & (q.x < 3.0 + w)).all()
    back = join_particles(parts, nx)
    order = lambda a: np.lexsort((a.z, a.y, a.x))   # noqa: E731
    a, b = order(p), order(back)
    for k in Particles.NAMES:
        np.testing.assert_array_equal(getattr(p, k)[a], getattr(back, k)[b])   # the integer shift is exact
    shape = (nx + 5, ny + 5, nz + 5)
    f = Fields(*(np.asfortranarray(rng.normal(size=shape)) for _ in range(6)))
    fs = split_fields(f, nx, S)
    for s, q in enumerate(fs):
        assert q.Ex.shape == (w + 5, ny + 5, nz + 5)
        np.testing.assert_array_equal(q.Ex[2:-3], f.Ex[2 + s * w:2 + (s + 1) * w])
        np.testing.assert_array_equal(q.Bz[:2], f.Bz[s * w:s * w + 2])        # ghosts = the neighbour's edge
    np.testing.assert_array_equal(join_interior(fs, "Ey"), f.Ey[2:-3])
