"""One periodic domain split along x into slabs: the reference's MPI
decomposition (src/comm/comm_fld.F90, comm_prtl.F90, loadprtlout.F90,
subdomains.F90:592-612, 720-740) restricted to x, on one GPU per slab.

Each slab is a ``Simulation`` with ``slab_x = 1`` holding nx / S interior
cells along x (y and z whole and periodic on the slab).  Its kernels leave
the x ghost layers and the particles leaving through the x faces to the
exchanges here, which run between the phases of the step exactly where
MAIN.F90 calls SendRecvFlds, ExchangePrtl and UpdateCurrentAllFaces:

    B half step, B faces | move + deposit, particles through the x faces |
    B half step, B faces | E update | J faces (ghost current added onto the
    neighbours' interior), y/z fold, AddCurrent, E faces | reorder

A ``Transport`` moves the face buffers: ``DistTransport`` between ranks
(torch.distributed point-to-point, NCCL between GPUs over NVLink, gloo on
CPU), ``LocalTransport`` between slabs that share a process (device
copies).  The left neighbour of slab 0 is slab S-1 (the periodic x axis).

A cylindrical domain (FP64, theta-gridded) splits along r the same way: slab
0 holds the axis (``inc_axis``), slab s starts at r = rmin + s w, and the
last slab's high face is the outer radius (``slab_x = 2``).  Those two
faces have no neighbour: the library drops what leaves through them and
neither packs nor unpacks them, so the ring transports carry the chain
unchanged (what slab 0 and slab S-1 exchange across the ring's seam is
ignored on both sides).
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from ._capi import check
from .simulation import Fields, Particles, PicConfig, Simulation

P_WORDS = 8   # doubles per particle in flight: q, x, y, z, u, v, w, flv
FIELD_NAMES = ("Ex", "Ey", "Ez", "Bx", "By", "Bz")


# ---------------------------------------------------------------------------
# transports
# ---------------------------------------------------------------------------
class LocalTransport:
    """All slabs of the ring in this process: what slab s sends right is
    what slab s+1 receives from the left (copies, on the tensors' device)."""

    def exchange(self, sends, recvs):
        """sends[s] = (to_left, to_right), recvs[s] = (from_left, from_right)
        for every slab s of the ring, in ring order."""
        n = len(sends)
        for s in range(n):
            recvs[s][0].copy_(sends[(s - 1) % n][1])
            recvs[s][1].copy_(sends[(s + 1) % n][0])

    def exchange_counts(self, counts):
        """counts[s] = (to_left, to_right) -> [(from_left, from_right)]."""
        n = len(counts)
        return [(counts[(s - 1) % n][1], counts[(s + 1) % n][0]) for s in range(n)]


class DistTransport:
    """One slab per rank of the default process group, ring neighbours
    rank - 1 (left) and rank + 1 (right).  Point-to-point pairs match in the
    order they are issued: every rank sends right then left and receives
    from the left then from the right, which pairs each rank's to_right
    with its right neighbour's from_left also when the two neighbours are
    the same rank (2 ranks)."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.left = (self.rank - 1) % self.world
        self.right = (self.rank + 1) % self.world

    def _pairs(self, to_left, to_right, from_left, from_right):
        if self.world == 1:
            if from_left is not None:
                from_left.copy_(to_right)
            if from_right is not None:
                from_right.copy_(to_left)
            return
        d = self.dist
        ops = []
        if to_right is not None:
            ops.append(d.P2POp(d.isend, to_right, self.right, self.group))
        if to_left is not None:
            ops.append(d.P2POp(d.isend, to_left, self.left, self.group))
        if from_left is not None:
            ops.append(d.P2POp(d.irecv, from_left, self.left, self.group))
        if from_right is not None:
            ops.append(d.P2POp(d.irecv, from_right, self.right, self.group))
        if ops:
            for r in d.batch_isend_irecv(ops):
                r.wait()

    def exchange(self, sends, recvs):
        (to_left, to_right), = sends
        (from_left, from_right), = recvs
        self._pairs(to_left, to_right, from_left, from_right)

    def exchange_counts(self, counts):
        import torch

        (nl, nr), = counts
        dev = _transport_device(self.dist, self.group)
        t_l = torch.tensor([nl], dtype=torch.int64, device=dev)
        t_r = torch.tensor([nr], dtype=torch.int64, device=dev)
        f_l = torch.zeros(1, dtype=torch.int64, device=dev)
        f_r = torch.zeros(1, dtype=torch.int64, device=dev)
        self._pairs(t_l, t_r, f_l, f_r)
        return [(int(f_l.item()), int(f_r.item()))]


def _transport_device(dist, group):
    import torch

    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")


def exchange_particle_buffers(transport, outs, counts, make_buffer):
    """Variable-size exchange of the particles that left through the x
    faces: the counts first, then the payloads (nothing is sent where a count
    is zero, on both sides alike).  outs[s] = (to_left, to_right) buffers,
    counts[s] = (n_to_left, n_to_right); returns [(from_left, n_left),
    (from_right, n_right)] per slab, buffers from make_buffer(n)."""
    incoming = transport.exchange_counts(counts)
    recvs = []
    for (nl, nr) in incoming:
        recvs.append((make_buffer(nl) if nl else None, make_buffer(nr) if nr else None))
    sends = []
    for (tl, tr), (cl, cr) in zip(outs, counts):
        sends.append((tl if cl else None, tr if cr else None))
    if isinstance(transport, LocalTransport):
        n = len(sends)
        for s in range(n):
            fl, fr = recvs[s]
            if fl is not None:
                fl.copy_(sends[(s - 1) % n][1])
            if fr is not None:
                fr.copy_(sends[(s + 1) % n][0])
    else:
        (tl, tr), = sends
        (fl, fr), = recvs
        transport._pairs(tl, tr, fl, fr)
    return [((fl, nl), (fr, nr)) for (fl, fr), (nl, nr) in zip(recvs, incoming)]


# ---------------------------------------------------------------------------
# splitting a global state into slabs (host side)
# ---------------------------------------------------------------------------
def slab_width(nx: int, nslabs: int) -> int:
    if nslabs < 1 or nx % nslabs or nx // nslabs < 5:
        raise ValueError(f"nx = {nx} does not split into {nslabs} slabs of at least 5 cells")
    return nx // nslabs


def split_particles(p: Particles, nx: int, nslabs: int) -> list[Particles]:
    """Slab s takes the particles with global x in [3 + s w, 3 + (s+1) w),
    x shifted into its own coordinates (exactly: an integer shift)."""
    w = slab_width(nx, nslabs)
    x = np.asarray(p.x)
    idx = np.clip(np.floor((x - 3.0) / w).astype(np.int64), 0, nslabs - 1)
    out = []
    for s in range(nslabs):
        m = idx == s
        fields = {k: np.ascontiguousarray(getattr(p, k)[m]) for k in Particles.NAMES}
        fields["x"] = fields["x"] - float(s * w)
        out.append(Particles(**fields))
    return out


def join_particles(parts: list[Particles], nx: int) -> Particles:
    """The slabs' live particles in global coordinates."""
    w = nx // len(parts)
    keep = []
    for s, p in enumerate(parts):
        m = np.asarray(p.flv) != 0
        f = {k: np.asarray(getattr(p, k))[m] for k in Particles.NAMES}
        f["x"] = f["x"] + float(s * w)
        keep.append(f)
    return Particles(**{k: np.concatenate([f[k] for f in keep]) for k in Particles.NAMES})


def split_fields(f: Fields, nx: int, nslabs: int) -> list[Fields]:
    """Slab s's ghosted arrays: global x indices s w + 1 .. s w + w + 5 (its
    ghosts are its neighbours' edge layers or the global periodic images)."""
    w = slab_width(nx, nslabs)
    out = []
    for s in range(nslabs):
        x0 = s * w
        out.append(Fields(*(np.asfortranarray(getattr(f, k)[x0:x0 + w + 5]) for k in FIELD_NAMES)))
    return out


def join_interior(parts: list[Fields], name: str) -> np.ndarray:
    """Interior x layers of every slab, in global order (y, z ghosted)."""
    return np.concatenate([getattr(p, name)[2:-3] for p in parts], axis=0)


# ---------------------------------------------------------------------------
# slabs and the step
# ---------------------------------------------------------------------------
class Slab:
    """One slab: a slab-form Simulation and its device exchange buffers."""

    def __init__(self, cfg: PicConfig, index: int, nslabs: int, device=None, out_capacity: int | None = None):
        import torch

        self.index, self.nslabs = index, nslabs
        self.w = slab_width(cfg.nx, nslabs)
        self.x0 = index * self.w
        if cfg.geom == "cylindrical":
            # r of the slab's first cell; the axis on slab 0, the outer radius on the last
            self.cfg = dataclasses.replace(cfg, nx=self.w, slab_x=2 if index == nslabs - 1 else 1,
                                           rmin=cfg.rmin + self.x0, inc_axis=cfg.inc_axis if index == 0 else 0)
        else:
            self.cfg = dataclasses.replace(cfg, nx=self.w, slab_x=1)
        self.sim = Simulation(self.cfg)
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        n = C.c_int64()
        check(self.sim.L.pic_slab_face_len(self.sim.h, C.byref(n)), "pic_slab_face_len")
        mk = lambda: torch.zeros(n.value, dtype=torch.float64, device=self.device)   # noqa: E731
        self.to_left, self.to_right, self.from_left, self.from_right = mk(), mk(), mk(), mk()
        # particles leaving through the x faces in one step, at most: those of
        # the two edge layers (a move is below one cell), capacity / w per
        # layer at the configured fill, with a factor 2 for the fluctuations
        self.out_capacity = int(out_capacity or 4 * (self.cfg.capacity // self.w) + 4096)
        self.out = torch.zeros(P_WORDS * self.out_capacity, dtype=torch.float64, device=self.device)
        self._boxes = None

    def boxes(self):
        """The fixed-size particle boxes (to_left, to_right, from_left,
        from_right): out_capacity particles and a count record each."""
        import torch

        if self._boxes is None:
            n = P_WORDS * (self.out_capacity + 1)
            self._boxes = tuple(torch.zeros(n, dtype=torch.float64, device=self.device) for _ in range(4))
        return self._boxes

    def close(self):
        self.sim.close()

    # faces --------------------------------------------------------------
    def pack_fields(self, which: int):
        check(self.sim.L.pic_slab_pack_fields(self.sim.h, which, self.to_left.data_ptr(), self.to_right.data_ptr()),
              "pic_slab_pack_fields")

    def unpack_fields(self, which: int):
        check(self.sim.L.pic_slab_unpack_fields(self.sim.h, which, self.from_left.data_ptr(),
                                                self.from_right.data_ptr()), "pic_slab_unpack_fields")

    def pack_particles(self):
        """-> ((to_left, n_left), (to_right, n_right)): views of the outbox."""
        nr, nl = C.c_int64(), C.c_int64()
        check(self.sim.L.pic_slab_pack_particles(self.sim.h, self.out.data_ptr(), self.out_capacity, C.byref(nr),
                                                 C.byref(nl)), "pic_slab_pack_particles")
        nr, nl = nr.value, nl.value
        to_right = self.out[:P_WORDS * nr]
        to_left = self.out[P_WORDS * nr:P_WORDS * (nr + nl)]
        return (to_left, nl), (to_right, nr)

    def unpack_particles(self, buf, n: int):
        if n:
            check(self.sim.L.pic_slab_unpack_particles(self.sim.h, buf.data_ptr(), int(n)),
                  "pic_slab_unpack_particles")

    def pack_particles_fixed(self):
        tl, tr, _, _ = self.boxes()
        check(self.sim.L.pic_slab_pack_particles_fixed(self.sim.h, tl.data_ptr(), tr.data_ptr(), self.out_capacity),
              "pic_slab_pack_particles_fixed")

    def unpack_particles_fixed(self):
        _, _, fl, fr = self.boxes()
        check(self.sim.L.pic_slab_unpack_particles_fixed(self.sim.h, fl.data_ptr(), fr.data_ptr(), self.out_capacity),
              "pic_slab_unpack_particles_fixed")


class SlabDomain:
    """The slabs of this process and the transport between them: MAIN.F90's
    step with the x exchanges (all slabs of the ring in one process with a
    LocalTransport, or one slab per rank with a DistTransport).

    queued=True: the library's phase calls only enqueue their work; a single
    slab's transfers run on its handle's stream (NCCL ordered after the pack
    kernels, the unpack kernels after the transfers), so a step waits on the
    host only for the particle counts; several slabs in one process
    synchronise the device around each exchange instead of after every
    call.

    fixed=True: the particles cross in fixed-size boxes that carry their
    counts (pic_slab_*_particles_fixed), so no count comes back to the host:
    queued with one slab, a step enqueues all its work and never waits."""

    E, B, J = 0, 1, 2

    def __init__(self, slabs: list[Slab], transport, queued: bool = False, fixed: bool = False):
        import torch

        self.slabs = slabs
        self.transport = transport
        self.t = 0
        self.queued = queued
        self.fixed = fixed
        self._stream = None
        if queued:
            for s in slabs:
                s.sim.set_sync(False)
            if len(slabs) == 1 and slabs[0].device.type == "cuda":
                self._stream = torch.cuda.ExternalStream(slabs[0].sim.stream, device=slabs[0].device)

    def _device_sync(self):
        import torch

        if self.slabs and self.slabs[0].device.type == "cuda":
            torch.cuda.synchronize(self.slabs[0].device)

    def _transfer(self, fn):
        """Run a transfer: on the slab's stream when queued with one slab,
        else between device synchronisations."""
        import torch

        if self._stream is not None:
            with torch.cuda.stream(self._stream):
                return fn()
        if self.queued:
            self._device_sync()
        r = fn()
        self._device_sync()
        return r

    def exchange_fields(self, which: int):
        for s in self.slabs:
            s.pack_fields(which)
        self._transfer(lambda: self.transport.exchange([(s.to_left, s.to_right) for s in self.slabs],
                                                       [(s.from_left, s.from_right) for s in self.slabs]))
        for s in self.slabs:
            s.unpack_fields(which)

    def exchange_particles(self):
        import torch

        if self.fixed:
            for s in self.slabs:
                s.pack_particles_fixed()
            self._transfer(lambda: self.transport.exchange([s.boxes()[:2] for s in self.slabs],
                                                           [s.boxes()[2:] for s in self.slabs]))
            for s in self.slabs:
                s.unpack_particles_fixed()
            return
        packed = [s.pack_particles() for s in self.slabs]
        outs = [(tl, tr) for (tl, _), (tr, _) in packed]
        counts = [(nl, nr) for (_, nl), (_, nr) in packed]
        dev = self.slabs[0].device
        got = self._transfer(lambda: exchange_particle_buffers(
            self.transport, outs, counts, lambda n: torch.empty(P_WORDS * n, dtype=torch.float64, device=dev)))
        # AppendParticles order: what came from the left, then from the right
        for s, ((fl, nl), (fr, nr)) in zip(self.slabs, got):
            s.unpack_particles(fl, nl)
            s.unpack_particles(fr, nr)

    def step(self, nsteps: int = 1):
        for _ in range(nsteps):
            self.t += 1
            for s in self.slabs:
                s.sim.update_b_half()
            self.exchange_fields(self.B)
            for s in self.slabs:
                s.sim.move_deposit()
            self.exchange_particles()
            for s in self.slabs:
                s.sim.update_b_half()
            self.exchange_fields(self.B)
            for s in self.slabs:
                s.sim.update_e()
            self.exchange_fields(self.J)
            for s in self.slabs:
                s.sim.fold_current()
                s.sim.add_current()
            self.exchange_fields(self.E)
            period = self.slabs[0].cfg.reorder_period
            if period and self.t % period == 0:
                for s in self.slabs:
                    s.sim.reorder()

    def close(self):
        for s in self.slabs:
            s.close()


def local_domain(cfg: PicConfig, nslabs: int, device=None, out_capacity: int | None = None,
                 queued: bool = False, fixed: bool = False) -> SlabDomain:
    """All slabs of a domain split along x in this process (one GPU)."""
    return SlabDomain([Slab(cfg, s, nslabs, device, out_capacity) for s in range(nslabs)], LocalTransport(), queued,
                      fixed)


def distributed_slab(cfg: PicConfig, group=None, out_capacity: int | None = None, queued: bool = True,
                     fixed: bool = False) -> SlabDomain:
    """This rank's slab of a domain split along x over the ranks of the
    process group (one GPU per rank, the current CUDA device)."""
    t = DistTransport(group)
    return SlabDomain([Slab(cfg, t.rank, t.world, None, out_capacity)], t, queued, fixed)
