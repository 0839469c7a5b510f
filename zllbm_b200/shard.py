"""Slab sharding of a single-level lattice over several contexts (one per GPU): the counterpart of
the reference's MPI partition, which gives each rank a contiguous range of background Morton codes
(amr_project/mpi/mpi_manager.h:137-140) and exchanges a one-node halo per level sub-step
(amr_project/mpi/mpi_grid_communication.cpp:210-357).  Here each rank owns a contiguous slab of
planes of the last axis, so its populations stay one dense box and every halo is a whole plane;
ranks form a ring when that axis is periodic.

With the single-buffer AA pattern an even step reads and writes only a node's own slots, so a pair
of steps needs two exchanges per face (``zl_set_level_halo`` in ``include/zllbm_b200.h``):

* stage 0, after the even step: the populations a face's boundary plane sends across the face go
  to the neighbour's ghost plane;
* stage 1, after the odd step: the populations this slab's nodes wrote into a ghost plane go back
  to the neighbour's boundary plane.

``SlabSchedule`` runs that schedule for one rank over any slab with ``step()``, ``pack(face,
stage)`` and ``unpack(face, stage, buf)`` and any ``exchange(sends) -> recvs``: ``DeviceSlab`` (a
library context on this rank's GPU) with ``torch_exchange`` (NCCL point-to-point), or host models
over gloo in the CPU tests.  ``LocalRing`` runs the same schedule for several slabs held by one
process (several contexts on one GPU), routing the buffers directly.

With ``overlap`` (slabs with ``step_planes``, at least five planes) a step's exchange is left in
flight while the next step updates the planes that do not need it, and completed before the rest:

* even step: planes [2, n - 2) first (they read only slots the previous odd step's planes
  [1, n - 1) wrote), then the stage-1 halo of the previous step is unpacked, then planes 0, 1,
  n - 2, n - 1 (which read the unpacked boundary slots or the slots of the boundary planes'
  previous odd update), then the stage-0 halo is packed and posted;
* odd step: planes [1, n - 1) first (no ghost plane is read or written there), then the stage-0
  halo is unpacked, then planes 0 and n - 1, then the stage-1 halo is packed and posted.

Every plane is updated exactly once per step and no update reads a slot that a later part of the
same step writes, so the result equals the unsplit schedule bit for bit; ``flush()`` completes the
last exchange (before reading the populations).
"""
from __future__ import annotations

from dataclasses import dataclass


def slab_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Planes [lo, hi) of `n` owned by `rank` of `world` (contiguous, sizes differing by at most one)."""
    if world < 1 or not 0 <= rank < world or n < world:
        raise ValueError(f"cannot split {n} planes over {world} ranks")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


@dataclass(frozen=True)
class Ring:
    """Neighbours of `rank` along the split axis; None at a closed end."""
    rank: int
    world: int
    periodic: bool

    @property
    def below(self):
        if self.rank > 0:
            return self.rank - 1
        return self.world - 1 if self.periodic else None

    @property
    def above(self):
        if self.rank < self.world - 1:
            return self.rank + 1
        return 0 if self.periodic else None

    @property
    def halo_faces(self) -> tuple[bool, bool]:
        """(low face, high face) of the split axis that are halo faces."""
        return self.below is not None, self.above is not None


class SlabSchedule:
    """Even step, stage-0 exchange, odd step, stage-1 exchange for one rank.

    `faces` = (low face, high face) of the split axis (face slots 2 axis, 2 axis + 1).
    `exchange(sends)` takes {peer: [buffers]} and returns {peer: [buffers]}: what each peer sent
    to this rank, in the order the peer listed them."""

    def __init__(self, slab, ring: Ring, faces: tuple[int, int], exchange, overlap: bool = False):
        self.slab = slab
        self.ring = ring
        self.lo_face, self.hi_face = faces
        self.exchange = exchange
        self.steps = 0
        self.overlap = overlap and plane_split_ok(slab)
        self.pending = None  # (stage, in-flight exchange) of the last step, overlap only

    def sends(self, stage: int) -> dict:
        """{peer: [buffers]}: the high face's buffer first (to the rank above), then the low face's."""
        out = {}
        if self.ring.above is not None:
            out.setdefault(self.ring.above, []).append(self.slab.pack(self.hi_face, stage))
        if self.ring.below is not None:
            out.setdefault(self.ring.below, []).append(self.slab.pack(self.lo_face, stage))
        return out

    def receive(self, stage: int, recvs: dict):
        """Unpack what the neighbours sent: the rank below sent its high face's buffer (for my low
        face) first in its list, the rank above its low face's buffer last."""
        if self.ring.below is not None:
            self.slab.unpack(self.lo_face, stage, recvs[self.ring.below][0])
        if self.ring.above is not None:
            self.slab.unpack(self.hi_face, stage, recvs[self.ring.above][-1])

    def swap(self, stage: int):
        self.receive(stage, self.exchange(self.sends(stage)))

    def step(self):
        """One time step and its exchange (stage 0 after an even step, stage 1 after an odd one)."""
        stage = self.steps & 1
        if not self.overlap:
            self.slab.step()
            self.steps += 1
            self.swap(stage)
            return
        inner, edges = plane_split(self.slab.n_planes, stage)
        self.slab.step_planes(*inner, False)
        self.flush()
        for k, (first, count) in enumerate(edges):
            self.slab.step_planes(first, count, k == len(edges) - 1)
        self.steps += 1
        self.pending = (stage, self.exchange.start(self.sends(stage)))

    def flush(self):
        """Complete the exchange still in flight (overlap only)."""
        if self.pending is not None:
            stage, handle = self.pending
            self.pending = None
            self.receive(stage, handle.wait())

    def step_pair(self):
        self.step()
        self.step()


def plane_split_ok(slab) -> bool:
    return hasattr(slab, "step_planes") and getattr(slab, "n_planes", 0) >= 5


def plane_split(n: int, stage: int):
    """((first, count) of the planes that do not wait for the exchange, [(first, count)] of the
    planes that do) for a step of parity `stage` on a slab of n planes."""
    if stage == 0:
        return (2, n - 4), [(0, 2), (n - 2, 2)]
    return (1, n - 2), [(0, 1), (n - 1, 1)]


class LocalRing:
    """The slab schedule for all ranks of a ring held by one process: every slab steps, packs,
    and unpacks what its neighbours packed (no collective; e.g. several contexts on one GPU).
    With overlap, the phases of the overlapped schedule run slab by slab in the same order."""

    def __init__(self, slabs, periodic: bool, faces: tuple[int, int], overlap: bool = False):
        world = len(slabs)
        self.scheds = [SlabSchedule(s, Ring(r, world, periodic), faces, None) for r, s in enumerate(slabs)]
        self.overlap = overlap and all(plane_split_ok(s) for s in slabs)
        self.pending = None  # (stage, sends of every slab)

    def _route(self, stage: int, sends):
        for r, s in enumerate(self.scheds):
            recvs = {peer: sends[peer][r] for peer in range(len(sends)) if r in sends[peer]}
            s.receive(stage, recvs)

    def step(self):
        """One time step of every slab (an even step swaps stage 0 after it, an odd one stage 1)."""
        stage = self.scheds[0].steps & 1
        if not self.overlap:
            for s in self.scheds:
                s.slab.step()
                s.steps += 1
            self._route(stage, [s.sends(stage) for s in self.scheds])
            return
        splits = [plane_split(s.slab.n_planes, stage) for s in self.scheds]
        for s, (inner, _) in zip(self.scheds, splits):
            s.slab.step_planes(*inner, False)
        self.flush()
        for s, (_, edges) in zip(self.scheds, splits):
            for k, (first, count) in enumerate(edges):
                s.slab.step_planes(first, count, k == len(edges) - 1)
            s.steps += 1
        self.pending = (stage, [s.sends(stage) for s in self.scheds])

    def flush(self):
        if self.pending is not None:
            stage, sends = self.pending
            self.pending = None
            self._route(stage, sends)

    def step_pair(self):
        self.step()
        self.step()


class _Posted:
    def __init__(self, reqs, recvs):
        self.reqs, self.recvs = reqs, recvs

    def wait(self) -> dict:
        for req in self.reqs:
            req.wait()
        return self.recvs


class TorchExchange:
    """exchange(sends) over torch.distributed point-to-point calls (NCCL for device tensors, gloo
    for host tensors).  Every rank sends as many buffers to a peer as it receives from it, of equal
    sizes (the neighbouring faces have the same plane), so each send is matched by a receive of
    the same shape posted in the same order.  start(sends) posts the exchange and returns a handle
    whose wait() gives the received buffers (for NCCL: the current stream then waits for the
    transfers, the host does not)."""

    def __init__(self, dist):
        self.dist = dist

    def start(self, sends: dict) -> _Posted:
        import torch
        dist = self.dist
        me = dist.get_rank()
        recvs, ops = {}, []
        for peer in sorted(sends):
            bufs = sends[peer]
            if peer == me:  # one-rank periodic ring: the high face wraps onto the low face
                recvs[peer] = [b.clone() for b in bufs]
                continue
            recvs[peer] = [torch.empty_like(b) for b in bufs]
            for b in bufs:
                ops.append(dist.P2POp(dist.isend, b, peer))
            for r in recvs[peer]:
                ops.append(dist.P2POp(dist.irecv, r, peer))
        return _Posted(dist.batch_isend_irecv(ops) if ops else [], recvs)

    def __call__(self, sends: dict) -> dict:
        return self.start(sends).wait()


def torch_exchange(dist) -> TorchExchange:
    return TorchExchange(dist)


def slab_config(config, lo: int, hi: int, ring: Ring):
    """The context configuration of planes [lo, hi) of the global configuration's last axis: the
    domain narrowed to the slab, and the faces toward neighbours made halo faces (no boundary
    condition; zl_set_level_halo connects them)."""
    import copy

    import zllbm_b200 as zl
    cfg = copy.deepcopy(config)
    axis = cfg.dims - 1
    kinds, dmin, dmax = list(cfg.bc_kind), list(cfg.domain_min), list(cfg.domain_max)
    g0 = dmin[axis]
    dmin[axis], dmax[axis] = g0 + lo, g0 + hi - 1
    below, above = ring.halo_faces
    if below:
        kinds[2 * axis] = zl.BC_NONE
    if above:
        kinds[2 * axis + 1] = zl.BC_NONE
    cfg.bc_kind, cfg.domain_min, cfg.domain_max = tuple(kinds), tuple(dmin), tuple(dmax)
    return cfg


def split_planes(config) -> int:
    """Planes of the global configuration's last axis (periodic: each plane once)."""
    import zllbm_b200 as zl
    axis = config.dims - 1
    span = config.domain_max[axis] - config.domain_min[axis]
    return span if config.bc_kind[2 * axis] == zl.BC_PERIODIC else span + 1


class DeviceSlab:
    """One rank's slab as a library context on the current GPU: a full box over planes [lo, hi)
    of the global configuration's last axis, halo faces where the ring has a neighbour.  Its node
    list `codes` is every node of the slab's domain the way the reference stores a level (the
    duplicated maximum plane of a periodic axis included), so populations and fields move without
    codes in that order.  Exchange buffers are torch uint8 device tensors of zl_halo_bytes."""

    def __init__(self, config, lo: int, hi: int, ring: Ring):
        import torch

        import zllbm_b200 as zl
        self.config = slab_config(config, lo, hi, ring)
        cfg = self.config
        dims = cfg.dims
        axis = dims - 1
        self.lo, self.hi = lo, hi
        self.faces = (2 * axis, 2 * axis + 1)
        self.ctx = zl.Context(cfg)
        # the context issues its work on torch's current stream, so that the exchange buffers
        # (allocated and sent by torch there) are ordered with the packs and unpacks; torch's
        # default stream is CUDA's legacy default stream, handle cudaStreamLegacy (1)
        self.ctx.set_stream(torch.cuda.current_stream().cuda_stream or 1)
        self.box_lo = tuple(cfg.domain_min[:dims])
        self.box_n = tuple(cfg.domain_max[a] - cfg.domain_min[a] + (0 if cfg.bc_kind[2 * a] == zl.BC_PERIODIC else 1)
                           for a in range(dims))
        self.codes = zl.box_codes(dims, cfg.domain_min[:dims], cfg.domain_max[:dims])
        self.ctx.set_level_nodes(0, self.codes)
        below, above = ring.halo_faces
        self.ctx.set_level_halo(0, (below << self.faces[0]) | (above << self.faces[1]))
        self.nbytes = {f: self.ctx.halo_bytes(0, f) for f in self.faces}

    def step(self):
        self.ctx.step_level(0)

    @property
    def n_planes(self) -> int:
        """Planes of the split axis (plane-range steps are D3Q19 only)."""
        return self.box_n[-1] if self.config.dims == 3 else 0

    def step_planes(self, first: int, count: int, finish: bool):
        self.ctx.step_level_planes(0, first, count, finish)

    def pack(self, face: int, stage: int):
        import torch
        buf = torch.empty(self.nbytes[face], dtype=torch.uint8, device="cuda")
        self.ctx.halo_pack(0, face, stage, buf.data_ptr())
        return buf

    def unpack(self, face: int, stage: int, buf):
        self.ctx.halo_unpack(0, face, stage, buf.data_ptr())

    def close(self):
        self.ctx.close()
