"""A vertex set replaced between steps (a body with prescribed motion, or a new set of areas):
nodes that only the previous set's stencils touched drop the force they last received, nodes of
an unchanged set keep theirs, and an emptied set leaves no force behind.  The node forces are
read back through the checkpoint writer (FP64 storage, forcing on)."""
import os

import numpy as np
import pytest

from oracle.checkpoint import parse
from test_gpu_amr import config, load_amr

pytestmark = pytest.mark.gpu


def node_forces(ctx, z, path):
    ctx.write_checkpoint_nodes(path, [z["codes0"]], [z["flags0"]])
    rec, n_forces = parse(open(path, "rb").read(), 9)
    assert n_forces == 2
    os.remove(path)
    return np.sort(rec, order="code")["force"].copy()


def test_moved_vertex_set_releases_old_stencil_forces(tmp_path):
    import zllbm_b200 as zl
    meta, z = load_amr("ib2d_l0")
    path = str(tmp_path / "grid_nodes")
    v = z["vertices_before"]
    xyz, area = v[:, 0:3].copy(), v[:, 6].copy()
    # a body with prescribed motion in a fluid at rest: F = 2 (U_b - u) is non-zero from the first pass
    uvw = np.zeros_like(xyz)
    uvw[:, 0], uvw[:, 1] = 0.02, 0.01
    moved = xyz.copy()
    moved[:, 0] -= 12.0  # stencils of the moved circle and of the old one share no node
    with zl.Context(config(meta, zl.STORAGE_F64)) as ctx:
        ctx.set_level_nodes(0, z["codes0"])
        ctx.set_populations(0, z["codes0"], z["f_before0"])
        ctx.ib_set_vertices(0, xyz, uvw, area)
        ctx.advance(2)
        before = node_forces(ctx, z, path)
        touched = np.abs(before).sum(1) > 0
        assert touched.sum() > 0

        # the same set again: every node keeps its force
        ctx.ib_set_vertices(0, xyz, uvw, area)
        assert np.array_equal(node_forces(ctx, z, path), before)

        # a moved set: the old band is released, the new one is forced by the next pass only
        ctx.ib_set_vertices(0, moved, uvw, area)
        assert not np.any(node_forces(ctx, z, path))
        ctx.advance(1)
        after = node_forces(ctx, z, path)
        moved_band = np.abs(after).sum(1) > 0
        assert moved_band.sum() > 0 and np.all(np.isfinite(after))
        assert not np.any(moved_band & touched)

        # an emptied set leaves no force behind
        ctx.ib_set_vertices(0, np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0))
        assert not np.any(node_forces(ctx, z, path))
