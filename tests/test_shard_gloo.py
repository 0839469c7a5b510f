"""Slab sharding (zllbm_b200.shard) on CPU: a host model of one slab's AA population slots with
ghost planes, whose halo pack / unpack follow the rule of zl_halo_pack / zl_halo_unpack, run
through the sharding schedule

* over gloo ranks (world size 2, where both neighbours are one peer, and 3, ragged slabs), in a
  periodic ring and in an open chain;
* in one process (LocalRing) and as a one-rank periodic ring exchanging with itself;
* with the overlapped schedule (interior planes stepped while the halo is in flight, the rest
  after it arrives) as well as the plain one;

and compared bit for bit with the global lattice stepped by plain collide-and-stream (two
buffers, periodic or open ends where a missing upstream node leaves the stale value, the rule of
a face without a boundary condition)."""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from oracle.port import LATTICE_C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
C = np.array(LATTICE_C[3], dtype=np.int64)
Q = len(C)
OPP = np.array([int(np.where((C == -c).all(1))[0][0]) for c in C])
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
SHAPE = (6, 5, 11)  # x, y, z nodes of the global lattice; z is split
SHAPE_OVERLAP = (6, 5, 21)  # at least five planes per slab for up to four slabs
TAU = 0.8
STEPS = 6


def collide(f):
    """BGK on populations f[q, ...] (any node-local map would do; this one mixes all of them)."""
    rho = f.sum(0)
    u = np.tensordot(C.T.astype(np.float64), f, axes=(1, 0)) / rho
    usq = (u * u).sum(0)
    out = np.empty_like(f)
    for q in range(Q):
        cu = np.tensordot(C[q].astype(np.float64), u, axes=(0, 0))
        feq = W[q] * rho * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * usq)
        out[q] = f[q] - (f[q] - feq) / TAU
    return out


def initial(seed=3, shape=SHAPE):
    """Populations f[q, z, y, x] near rest with a seeded perturbation."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    return W[:, None, None, None] * (1 + 0.05 * rng.standard_normal((Q, nz, ny, nx)))


def two_buffer(f, steps, periodic_z):
    """Collide, then stream f(x + c_q, q) = f*(x, q); x and y periodic, z periodic or open (a node
    whose upstream node is missing keeps its pre-collision value)."""
    nz = f.shape[1]
    for _ in range(steps):
        post = collide(f)
        new = np.empty_like(f)
        for q in range(Q):
            cx, cy, cz = C[q]
            moved = np.roll(post[q], (cz, cy, cx), axis=(0, 1, 2))
            if not periodic_z and cz:
                stale = 0 if cz > 0 else nz - 1  # the plane whose upstream plane is missing
                moved[stale] = f[q, stale]
            new[q] = moved
        f = new
    return f


class HostSlab:
    """Planes [lo, hi) of the z axis with one ghost plane each side; slot array F[q, z, y, x]
    holds the AA layout (even steps: own slots; odd steps: neighbour slots), x and y periodic.
    Faces: 4 (z low) and 5 (z high)."""

    def __init__(self, f_global, lo, hi, halo):
        import torch
        self.torch = torch
        self.halo = halo  # (low face, high face) connected to a neighbour
        nz = hi - lo
        self.n = nz
        self.F = np.zeros((Q, nz + 2) + f_global.shape[2:])
        self.F[:, 1:-1] = f_global[:, lo:hi]
        self.odd = False

    def _missing(self, q):
        """Interior planes (1-based slot z) whose upstream plane z - c_z is off a closed face."""
        cz = C[q, 2]
        if cz > 0 and not self.halo[0]:
            return [1]
        if cz < 0 and not self.halo[1]:
            return [self.n]
        return []

    @property
    def n_planes(self):
        return self.n

    def step(self):
        self.step_planes(0, self.n, True)

    def step_planes(self, first, count, finish):
        """The node updates of planes [first, first + count) with the current parity (slot z = 1 +
        plane); finish flips the parity.  Each node reads and writes only its own slot set."""
        F = self.F
        a, b = first + 1, first + count + 1  # slot range of the planes
        cx, cy, cz = C[:, 0], C[:, 1], C[:, 2]
        if count > 0 and not self.odd:
            pre = F[:, a:b].copy()
            post = collide(pre)
            for q in range(Q):
                F[OPP[q], a:b] = post[q]
            for q in range(1, Q):
                for z in self._missing(q):  # stale value into the slot of the missing upstream cell
                    if a <= z < b:
                        F[OPP[q], z - cz[q]] = np.roll(pre[q, z - a], (-cy[q], -cx[q]), axis=(0, 1))
        elif count > 0:
            pre = np.empty((Q, count) + F.shape[2:])
            for q in range(Q):
                if q == 0:
                    pre[q] = F[0, a:b]
                else:  # f(x, q) in slot (x - c_q, opp q)
                    src = F[OPP[q], a - cz[q]:b - cz[q]]
                    pre[q] = np.roll(src, (cy[q], cx[q]), axis=(1, 2))
            post = collide(pre)
            for q in range(Q):
                if q == 0:
                    F[0, a:b] = post[0]
                else:  # f*(x, q) into slot (x + c_q, q)
                    F[q, a + cz[q]:b + cz[q]] = np.roll(post[q], (cy[q], cx[q]), axis=(1, 2))
            for q in range(1, Q):
                for z in self._missing(q):
                    if a <= z < b:
                        F[q, z] = pre[q, z - a]
        if finish:
            self.odd = not self.odd

    # the halo rule of zl_halo_pack / zl_halo_unpack
    def _planes(self, face, inward):
        sign = (-1 if inward else 1) if face & 1 else (1 if inward else -1)
        return [q for q in range(Q) if C[q, 2] == sign]

    def _layer(self, face, ghost):
        hi = face & 1
        return (self.n + 1 if hi else 0) if ghost else (self.n if hi else 1)

    def pack(self, face, stage):
        planes = self._planes(face, inward=stage == 0)
        layer = self._layer(face, ghost=stage == 1)
        return self.torch.from_numpy(np.ascontiguousarray(self.F[planes, layer]))

    def unpack(self, face, stage, buf):
        planes = self._planes(face, inward=stage == 1)
        layer = self._layer(face, ghost=stage == 0)
        self.F[planes, layer] = buf.numpy()

    def populations(self):
        """f[q, z, y, x] of the slab's nodes (even step count: natural layout)."""
        assert not self.odd
        return self.F[:, 1:-1].copy()


def _reference(periodic, shape=SHAPE):
    return two_buffer(initial(shape=shape), STEPS, periodic)


def test_slab_range_covers_every_plane_once():
    from zllbm_b200.shard import slab_range
    for n, world in [(11, 3), (256, 8), (7, 7), (10, 4)]:
        spans = [slab_range(n, r, world) for r in range(world)]
        assert spans[0][0] == 0 and spans[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
        sizes = [hi - lo for lo, hi in spans]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        slab_range(3, 0, 4)


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_local_ring_matches_global_lattice(world, periodic, overlap):
    from zllbm_b200.shard import LocalRing, Ring, slab_range
    shape = SHAPE_OVERLAP if overlap else SHAPE
    f0 = initial(shape=shape)
    slabs = []
    for r in range(world):
        lo, hi = slab_range(shape[2], r, world)
        slabs.append(HostSlab(f0, lo, hi, Ring(r, world, periodic).halo_faces))
    ring = LocalRing(slabs, periodic, (4, 5), overlap=overlap)
    assert ring.overlap == overlap
    for _ in range(STEPS // 2):
        ring.step_pair()
    ring.flush()
    got = np.concatenate([s.populations() for s in slabs], axis=1)
    assert np.array_equal(got, _reference(periodic, shape))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, periodic, overlap, out):
    import sys

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from test_shard_gloo import SHAPE, SHAPE_OVERLAP, HostSlab, initial
    from zllbm_b200.shard import Ring, SlabSchedule, slab_range, torch_exchange
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        shape = SHAPE_OVERLAP if overlap else SHAPE
        lo, hi = slab_range(shape[2], rank, world)
        ring = Ring(rank, world, periodic)
        slab = HostSlab(initial(shape=shape), lo, hi, ring.halo_faces)
        sched = SlabSchedule(slab, ring, (4, 5), torch_exchange(dist), overlap=overlap)
        assert sched.overlap == overlap
        for _ in range(STEPS // 2):
            sched.step_pair()
        sched.flush()
        out.put((rank, lo, hi, slab.populations()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_match_global_lattice(world, periodic, overlap):
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, periodic, overlap, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted((out.get(timeout=180) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref = _reference(periodic, SHAPE_OVERLAP if overlap else SHAPE)
    for rank, lo, hi, f in results:
        assert np.array_equal(f, ref[:, lo:hi]), rank


@pytest.mark.parametrize("overlap", [False, True])
def test_one_rank_ring_exchanges_with_itself(overlap):
    """A periodic ring of one rank: its high face's buffers wrap onto its own low face."""
    from zllbm_b200.shard import Ring, SlabSchedule

    class Dist:
        @staticmethod
        def get_rank():
            return 0

    from zllbm_b200.shard import torch_exchange
    ring = Ring(0, 1, True)
    shape = SHAPE_OVERLAP if overlap else SHAPE
    slab = HostSlab(initial(shape=shape), 0, shape[2], ring.halo_faces)
    sched = SlabSchedule(slab, ring, (4, 5), torch_exchange(Dist), overlap=overlap)
    for _ in range(STEPS // 2):
        sched.step_pair()
    sched.flush()
    assert np.array_equal(slab.populations(), _reference(True, shape))
