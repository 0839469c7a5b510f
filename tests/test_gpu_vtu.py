"""VTK XML field output built on the device (zl_write_vtu) against the reference's own writer.

The populations are the reference's state after its run (FP64 storage); the points are passed in
the order the reference wrote them.  The files must equal, byte for byte, the restatement in
oracle/vtu.py (pinned to the reference's files by test_vtu_oracle.py) with "rho" the density of
the current populations; every other array is checked against the reference's file directly."""
import json
import os

import numpy as np
import pytest

from fixtures import GOLDEN
from oracle import vtu
from test_gpu_amr import config
from test_vtu_oracle import reference_order

pytestmark = pytest.mark.gpu
CASES = ("tgv3d", "amr2d_l1", "force2d_mrt")


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("binary", [True, False])
def test_write_vtu_matches_reference(name, binary, tmp_path):
    import zllbm_b200 as zl
    z = np.load(os.path.join(GOLDEN, f"vtu_{name}.npz"))
    meta = json.loads(str(z["meta"]))
    dims, levels = meta["dims"], meta["levels"] + 1
    force = [float(v) for v in meta["cforce"].split(",")] if "cforce" in meta else None
    tag = "bin" if binary else "asc"
    order, expected = [], []
    for lv in range(levels):
        ref = bytes(z[f"vtu_{tag}{lv}"])
        codes, pos = reference_order(z, lv, dims, ref)
        rho, vel = vtu.output_macros(z[f"f{lv}"][pos], dims, force, dt=1.0 / (1 << lv))
        coords = vtu.coordinates(codes, dims, lv, (1.0, 1.0, 1.0), (-1.0, -1.0, -1.0))
        expected.append(vtu.level_vtu(binary, dims, z[f"flags{lv}"][pos], rho, vel, coords, vtu.cells(codes, dims)))
        order.append((codes, z[f"flags{lv}"][pos]))
    prefix = str(tmp_path / "run")
    with zl.Context(config(meta, zl.STORAGE_F64)) as ctx:
        for lv in range(levels):
            ctx.set_level_nodes(lv, z[f"codes{lv}"])
            ctx.set_populations(lv, z[f"codes{lv}"], z[f"f{lv}"])
        ctx.write_vtu(prefix, [c for c, _ in order], [f for _, f in order], binary=binary)
    for lv in range(levels):
        got = open(f"{prefix}_data/rank_0_grid_level_{lv}.vtu", "rb").read()
        assert got == expected[lv], f"level {lv}"
        mine, theirs = vtu.parse_arrays(got), vtu.parse_arrays(bytes(z[f"vtu_{tag}{lv}"]))
        assert mine.keys() == theirs.keys()
        for key in mine:
            if key != "rho":
                assert np.array_equal(mine[key][2], theirs[key][2]), key
    assert open(f"{prefix}_data/rank_0_.pvtu", "rb").read() == bytes(z[f"pvtu_{tag}"])


def test_write_vtu_reduced_storage_velocity(tmp_path):
    # FP32 storage: the same layout, velocity within FP32 rounding of the FP64 values
    import zllbm_b200 as zl
    z = np.load(os.path.join(GOLDEN, "vtu_tgv3d.npz"))
    meta = json.loads(str(z["meta"]))
    ref = bytes(z["vtu_bin0"])
    codes, pos = reference_order(z, 0, 3, ref)
    prefix = str(tmp_path / "run")
    with zl.Context(config(meta, zl.STORAGE_F32)) as ctx:
        ctx.set_level_nodes(0, z["codes0"])
        ctx.set_populations(0, z["codes0"], z["f0"])
        ctx.write_vtu(prefix, [codes], [z["flags0"][pos]])
    mine = vtu.parse_arrays(open(f"{prefix}_data/rank_0_grid_level_0.vtu", "rb").read())
    theirs = vtu.parse_arrays(ref)
    np.testing.assert_allclose(mine["velocity"][2], theirs["velocity"][2], rtol=0, atol=1e-7)
    for key in ("flag_status", "vtkGhostType", "Points", "connectivity", "offsets", "types"):
        assert np.array_equal(mine[key][2], theirs[key][2]), key


def test_write_vtu_rejects_foreign_codes(tmp_path):
    import zllbm_b200 as zl
    z = np.load(os.path.join(GOLDEN, "vtu_tgv3d.npz"))
    meta = json.loads(str(z["meta"]))
    with zl.Context(config(meta, zl.STORAGE_F64)) as ctx:
        ctx.set_level_nodes(0, z["codes0"])
        bad = np.array([np.uint64(1) << np.uint64(40)], dtype=np.uint64)
        with pytest.raises(zl.ZlError):
            ctx.write_vtu(str(tmp_path / "bad"), [bad], [np.zeros(1, np.int32)])
