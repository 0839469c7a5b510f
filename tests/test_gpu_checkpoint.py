"""Checkpoint node records from and into the device (zl_write_checkpoint_nodes /
zl_read_checkpoint_nodes) against the files the reference's own writer produced: FP64 storage
writes them byte for byte and reads them back bit for bit."""
import glob
import json
import os

import numpy as np
import pytest

from fixtures import GOLDEN
from test_gpu_amr import config

pytestmark = pytest.mark.gpu
CASES = sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN, "ckpt_*.npz")))


def _ctx(meta, z, storage):
    import zllbm_b200 as zl
    ctx = zl.Context(config(meta, storage))
    for lv in range(meta["levels"] + 1):
        ctx.set_level_nodes(lv, z[f"codes{lv}"])
    return ctx


@pytest.mark.parametrize("name", CASES)
def test_write_checkpoint_matches_reference(name, tmp_path):
    import zllbm_b200 as zl
    z = np.load(os.path.join(GOLDEN, f"ckpt_{name}.npz"))
    meta = json.loads(str(z["meta"]))
    levels = range(meta["levels"] + 1)
    path = str(tmp_path / "grid_nodes")
    with _ctx(meta, z, zl.STORAGE_F64) as ctx:
        for lv in levels:
            ctx.set_populations(lv, z[f"codes{lv}"], z[f"f{lv}"])
        ctx.write_checkpoint_nodes(path, [z[f"codes{lv}"] for lv in levels], [z[f"flags{lv}"] for lv in levels])
    assert open(path, "rb").read() == z["grid_nodes"].tobytes()


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("storage", [0, 1])
def test_read_checkpoint_restores_populations(name, storage, tmp_path):
    import zllbm_b200 as zl
    z = np.load(os.path.join(GOLDEN, f"ckpt_{name}.npz"))
    meta = json.loads(str(z["meta"]))
    path = str(tmp_path / "grid_nodes")
    z["grid_nodes"].tofile(path)
    with _ctx(meta, z, storage) as ctx:
        ctx.read_checkpoint_nodes(path)
        for lv in range(meta["levels"] + 1):
            got = ctx.get_populations(lv, z[f"codes{lv}"])
            if storage == zl.STORAGE_F64:
                assert np.array_equal(got, z[f"f{lv}"])
            else:
                np.testing.assert_allclose(got, z[f"f{lv}"], rtol=0, atol=1e-7)
