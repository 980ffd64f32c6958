"""The slab step on CPU with 3 gloo ranks: SlabDomain's phase and exchange
sequence (B faces twice, particles through the x faces with counts first,
the ghost current added onto the neighbours, E faces) driven through the
ring transport, on a 1-D stand-in for the library's slab (the same face
layers and buffer layouts, dyadic arithmetic so that every sum is exact).
Three slabs over three ranks give exactly the single periodic domain."""
import os
import socket
from types import SimpleNamespace

import numpy as np
import torch.multiprocessing as mp

NX, W_STEPS, PERIOD = 24, 6, 4


class ToySim:
    """1-D fields E, B, J on w interior cells with 2 low and 3 high ghost
    layers (the library's x layout) and particles (x, u, q); the phase
    methods SlabDomain calls."""

    def __init__(self, w, E, B, parts):
        self.w, self.m = w, w + 5
        self.E, self.B, self.J = E.copy(), B.copy(), np.zeros(w + 5)
        self.p = [list(q) for q in parts]          # [q, x, u]

    def update_b_half(self):
        i = np.arange(2, self.w + 2)
        self.B[i] = self.B[i] + (self.E[i + 1] - self.E[i]) / 2

    def move_deposit(self):
        self.J[:] = 0.0
        for q in self.p:
            q[1] = q[1] + q[2]
            self.J[int(np.floor(q[1])) - 1] += q[0]

    def update_e(self):
        i = np.arange(2, self.w + 2)
        self.E[i] = self.E[i] + (self.B[i] - self.B[i - 1])

    def fold_current(self):
        pass

    def add_current(self):
        i = np.arange(2, self.w + 2)
        self.E[i] = self.E[i] - self.J[i]

    def reorder(self):
        self.p.sort(key=lambda q: (q[1], q[2], q[0]))

    def set_sync(self, flag):
        pass


class ToySlab:
    """The Slab interface of pictor_b200.slab over a ToySim."""

    def __init__(self, w, E, B, parts):
        import torch

        self.sim = ToySim(w, E, B, parts)
        self.cfg = SimpleNamespace(reorder_period=PERIOD)
        self.device = torch.device("cpu")
        self.to_left, self.to_right, self.from_left, self.from_right = (torch.zeros(3, dtype=torch.float64)
                                                                        for _ in range(4))
        self.out = torch.zeros(8 * 256, dtype=torch.float64)

    def _field(self, which):
        return (self.sim.E, self.sim.B, self.sim.J)[which]

    def pack_fields(self, which):
        F, m = self._field(which), self.sim.m
        tl, tr = self.to_left.numpy(), self.to_right.numpy()
        if which == 2:                    # ghost current leaves: {1,2} left, {m-2..m} right
            tl[:2], tr[:3] = F[0:2], F[m - 3:m]
            F[0:2] = 0.0
            F[m - 3:m] = 0.0
        else:                             # interior {3,4,5} left, {m-4,m-3} right
            tl[:3], tr[:2] = F[2:5], F[m - 5:m - 3]

    def unpack_fields(self, which):
        F, m = self._field(which), self.sim.m
        fl, fr = self.from_left.numpy(), self.from_right.numpy()
        if which == 2:
            F[2:5] = F[2:5] + fl[:3]
            F[m - 5:m - 3] = F[m - 5:m - 3] + fr[:2]
        else:
            F[0:2] = fl[:2]
            F[m - 3:m] = fr[:3]

    def pack_particles(self):
        w = self.sim.w
        right = [q for q in self.sim.p if q[1] >= w + 3]
        left = [q for q in self.sim.p if q[1] < 3]
        self.sim.p = [q for q in self.sim.p if 3 <= q[1] < w + 3]
        o = self.out.numpy()
        for n, q in enumerate(right + left):
            x = q[1] - w if n < len(right) else q[1] + w
            o[8 * n:8 * n + 8] = [q[0], x, 0, 0, q[2], 0, 0, 1]
        nr, nl = len(right), len(left)
        return (self.out[8 * nr:8 * (nr + nl)], nl), (self.out[:8 * nr], nr)

    def unpack_particles(self, buf, n):
        if n:
            a = buf.numpy().reshape(n, 8)
            self.sim.p += [[r[0], r[1], r[4]] for r in a]

    def close(self):
        pass


def _initial(seed=5):
    rng = np.random.default_rng(seed)
    m = NX + 5
    E = rng.integers(-64, 64, m) / 64.0
    B = rng.integers(-64, 64, m) / 64.0
    E[0:2], E[m - 3:m] = E[m - 5:m - 3], E[2:5]          # periodic images
    B[0:2], B[m - 3:m] = B[m - 5:m - 3], B[2:5]
    parts = [[rng.integers(1, 8) / 8.0, 3 + rng.integers(0, 64 * NX) / 64.0, rng.integers(-56, 57) / 64.0]
             for _ in range(300)]
    return E, B, parts


def _split(E, B, parts, S, s):
    w = NX // S
    x0 = s * w
    mine = [[q, x - x0, u] for q, x, u in parts if x0 + 3 <= x < x0 + w + 3]
    return ToySlab(w, E[x0:x0 + w + 5], B[x0:x0 + w + 5], mine)


def _result(slab, S, s):
    w = NX // S
    x0 = s * w
    return (slab.sim.E[2:w + 2].copy(), slab.sim.B[2:w + 2].copy(),
            sorted((q, x + x0, u) for q, x, u in slab.sim.p))


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from pictor_b200.slab import DistTransport, SlabDomain

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    E, B, parts = _initial()
    slab = _split(E, B, parts, world, rank)
    dom = SlabDomain([slab], DistTransport())
    dom.step(W_STEPS)
    res = _result(slab, world, rank)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, res))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_three_rank_slabs_equal_single_domain():
    from pictor_b200.slab import LocalTransport, SlabDomain

    E, B, parts = _initial()
    one = _split(E, B, parts, 1, 0)
    SlabDomain([one], LocalTransport()).step(W_STEPS)
    E1, B1, P1 = _result(one, 1, 0)
    world = 3
    ctx = mp.get_context("spawn")
    qu = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, qu)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(qu.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    E3 = np.concatenate([out[r][0] for r in range(world)])
    B3 = np.concatenate([out[r][1] for r in range(world)])
    P3 = sorted(sum((out[r][2] for r in range(world)), []))
    np.testing.assert_array_equal(E3, E1)
    np.testing.assert_array_equal(B3, B1)
    assert len(P3) == len(P1) == 300
    np.testing.assert_array_equal(np.array(P3), np.array(P1))
    # the toy moved particles across the slab faces and through the periodic one
    assert any(x < 3 + NX // 3 for _, x, _ in P1) and any(x >= 3 + 2 * NX // 3 for _, x, _ in P1)
