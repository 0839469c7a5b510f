"""The restated order and layout of the reference's checkpoint node records (oracle/checkpoint.py)
reproduce, byte for byte, the grid_nodes files the reference's own writer produced."""
import glob
import json
import os

import numpy as np
import pytest

from fixtures import GOLDEN

CASES = sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN, "ckpt_*.npz")))


@pytest.mark.parametrize("name", CASES)
def test_restated_checkpoint_matches_reference_bytes(name):
    from oracle import checkpoint as ck
    z = np.load(os.path.join(GOLDEN, f"ckpt_{name}.npz"))
    meta = json.loads(str(z["meta"]))
    dims = meta["dims"]
    q = 9 if dims == 2 else 19
    raw = z["grid_nodes"].tobytes()
    rec, n_forces = ck.parse(raw, q)
    levels = [dict(codes=z[f"codes{lv}"], flags=z[f"flags{lv}"], f=z[f"f{lv}"]) for lv in range(meta["levels"] + 1)]
    assert ck.grid_nodes(dims, levels, n_forces) == raw
    assert rec.size == sum(lv["codes"].size for lv in levels)
    assert n_forces == (dims if "cforce" in meta else 0)


def test_cases_cover_levels_dims_and_forces():
    assert {"amr2d_l1", "amr3d_l1", "force2d_mrt", "force3d_srt"} <= set(CASES)
