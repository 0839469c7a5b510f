"""A CPU model of the step kernel's index maps (the AA pattern of aa_kernel.cuh: post_stream_slot,
post_collision_slot) on small periodic boxes: in each step every population slot is written
exactly once, each node reads and writes the same set of slots (so nodes need no ordering
between them: no races without synchronisation), and two AA steps equal two steps of the
reference's collide-then-pull-stream."""
import itertools

import numpy as np
import pytest

from oracle.port import LATTICE_C


def lattice(dims):
    c = np.array(LATTICE_C[dims], dtype=np.int64)
    opp = np.array([int(np.where((c == -ci).all(1))[0][0]) for ci in c])
    return c, opp


def slot(x, q, shape):
    """Flat slot index of plane q at (wrapped) cell x."""
    x = tuple(int(v) % s for v, s in zip(x, shape))
    return q * int(np.prod(shape)) + int(np.ravel_multi_index(x[::-1], shape[::-1]))


def aa_maps(dims, shape, even):
    """(reads, writes) per node for the even (own slots) or odd (neighbour slots) step: node x
    reads f(x, q) and writes f*(x, o)."""
    c, opp = lattice(dims)
    q_count = len(c)
    reads, writes = {}, {}
    for x in itertools.product(*[range(s) for s in shape]):
        x = np.array(x)
        if even:  # layout in: f(x, q) in slot (x, q); out: f*(x, o) in slot (x, opp o)
            r = [slot(x, q, shape) for q in range(q_count)]
            w = [slot(x, opp[o], shape) for o in range(q_count)]
        else:  # layout in: f(x, q) in slot (x - c_q, opp q); out: f*(x, o) in slot (x + c_o, o)
            r = [slot(x - c[q], opp[q], shape) for q in range(q_count)]
            w = [slot(x + c[o], o, shape) for o in range(q_count)]
        reads[tuple(x)], writes[tuple(x)] = r, w
    return reads, writes


def collide(x, f):
    """Any node-local map (depends on the node and all its populations); integers keep it exact."""
    q = len(f)
    return np.array([(f[(o * 7 + 3) % q] * 3 + f[o] + (o + 1) * (sum(x) + 1)) % 1000003 for o in range(q)],
                    dtype=np.int64)


@pytest.mark.parametrize("dims,shape", [(2, (5, 4)), (3, (4, 3, 5))])
def test_aa_write_sets_are_permutations_and_in_place(dims, shape):
    total = len(LATTICE_C[dims]) * int(np.prod(shape))
    for even in (True, False):
        reads, writes = aa_maps(dims, shape, even)
        every = [s for w in writes.values() for s in w]
        assert sorted(every) == list(range(total))  # each slot written exactly once per step
        for x in reads:
            assert sorted(reads[x]) == sorted(writes[x])  # a node touches only its own slot set


@pytest.mark.parametrize("dims,shape", [(2, (5, 4)), (3, (4, 3, 5))])
def test_two_aa_steps_equal_two_pull_steps(dims, shape):
    c, opp = lattice(dims)
    q_count = len(c)
    rng = np.random.default_rng(3)
    cells = list(itertools.product(*[range(s) for s in shape]))
    f0 = {x: rng.integers(0, 1000, q_count) for x in cells}

    # reference order: collide every node, then pull f(x, q) = f*(x - c_q, q) (periodic)
    ref = dict(f0)
    for _ in range(2):
        post = {x: collide(x, ref[x]) for x in cells}
        ref = {x: np.array([post[tuple((np.array(x) - c[q]) % shape)][q] for q in range(q_count)]) for x in cells}

    # AA: one buffer updated in place, even step then odd step, nodes in a shuffled order (the
    # kernel's blocks run in any order)
    buf = np.zeros(q_count * int(np.prod(shape)), dtype=np.int64)
    for x in cells:
        for q in range(q_count):
            buf[slot(x, q, shape)] = f0[x][q]
    for even in (True, False):
        reads, writes = aa_maps(dims, shape, even)
        for i in rng.permutation(len(cells)):
            x = cells[i]
            buf[writes[x]] = collide(x, buf[reads[x]])
    got = {x: buf[[slot(x, q, shape) for q in range(q_count)]] for x in cells}  # odd layout: (x, q)
    for x in cells:
        assert np.array_equal(got[x], ref[x])
