"""The VTK XML output restatement (oracle/vtu.py) against the reference's own writer: every
level's .vtu and the .pvtu, binary and ASCII, byte for byte."""
import json
import os

import numpy as np
import pytest

from oracle import vtu
from oracle.port import morton_encode

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ("tgv3d", "amr2d_l1", "force2d_mrt")


def reference_order(z, lv, dims, text):
    """Codes of the points in the order the reference wrote them (its hash-map order)."""
    pts = vtu.parse_arrays(text)["Points"][2].astype(np.float64).reshape(-1, 3)
    idx = np.rint((pts[:, :dims] + 1.0) * (1 << lv)).astype(np.int64)
    codes = morton_encode(idx, dims)
    pos = np.searchsorted(z[f"codes{lv}"], codes)
    assert np.array_equal(z[f"codes{lv}"][pos], codes)
    return codes, pos


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("binary", [True, False])
def test_vtu_restatement_matches_reference(name, binary):
    z = np.load(os.path.join(HERE, "golden", f"vtu_{name}.npz"))
    case = json.loads(str(z["meta"]))
    dims, levels = case["dims"], case["levels"] + 1
    force = [float(v) for v in case["cforce"].split(",")] if "cforce" in case else None
    tag = "bin" if binary else "asc"
    for lv in range(levels):
        ref = bytes(z[f"vtu_{tag}{lv}"])
        codes, pos = reference_order(z, lv, dims, ref)
        _, vel = vtu.output_macros(z[f"f{lv}"][pos], dims, force, dt=1.0 / (1 << lv))
        coords = vtu.coordinates(codes, dims, lv, (1.0, 1.0, 1.0), (-1.0, -1.0, -1.0))
        text = vtu.level_vtu(binary, dims, z[f"flags{lv}"][pos], z[f"rho_member{lv}"][pos], vel, coords,
                             vtu.cells(codes, dims))
        assert text == ref, f"level {lv}"
    assert vtu.pvtu(binary, dims, levels) == bytes(z[f"pvtu_{tag}"])


def test_vtu_cells_and_ghosts_present():
    # the multi-level case carries coarse/fine interface flags, hence ghost points, on both levels
    z = np.load(os.path.join(HERE, "golden", "vtu_amr2d_l1.npz"))
    for lv in range(2):
        arrays = vtu.parse_arrays(bytes(z[f"vtu_bin{lv}"]))
        assert arrays["vtkGhostType"][2].sum() > 0
        assert arrays["types"][2].size > 0 and np.all(arrays["types"][2] == 8)
        assert np.array_equal(arrays["offsets"][2], 4 * np.arange(1, arrays["types"][2].size + 1))
