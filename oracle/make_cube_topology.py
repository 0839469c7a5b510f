"""Node sets and interface layers of the multi-level cube-flow grid, generated by the reference's
own grid builder (refinement around a GeometryInfoOrigin cube, AmrManager::SetupMesh) through
the oracle harness, and saved as the input of ``python -m zllbm_b200.cube_flow``.

    python oracle/make_cube_topology.py OUT.npz [--n 256,128,128] [--levels 2] [--cube 80,64,64,16]
                                                [--ext 6] [--inner 16]

Needs the reference tree and ``make -C oracle ref``.  Per level l the archive holds the sorted
Morton codes and flag_status of its nodes; per refined level the explosion targets (the
level's coarse-to-fine layers), the coalescence targets on the level below and that level's
coarse-to-fine ghost nodes (excluded as explosion sources), exactly as the multi-level parity
tests feed them to zl_set_level_interface.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle.port import REF_RUN, load_levels  # noqa: E402


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("out")
    ap.add_argument("--n", default="256,128,128")
    ap.add_argument("--levels", type=int, default=2)
    ap.add_argument("--cube", default="80,64,64,16")
    ap.add_argument("--ext", default="6")
    ap.add_argument("--inner", default="16")
    a = ap.parse_args(argv)
    if not os.path.exists(REF_RUN):
        subprocess.run(["make", "-C", HERE, "ref"], check=True)
    meta = {"dims": 3, "n": [int(v) for v in a.n.split(",")], "levels": a.levels, "cube": a.cube,
            "ext": a.ext, "inner": a.inner}
    with tempfile.TemporaryDirectory() as tmp:
        dump = os.path.join(tmp, "l0.bin")
        subprocess.run([REF_RUN, "dims=3", f"n={a.n}", f"levels={a.levels}", f"geo=cube:{a.cube}", f"ext={a.ext}",
                        f"inner={a.inner}", "coll=srt", "nu=0.01", "steps=0", f"lout0={dump}",
                        "bc=xmin:neq:0.05,0,0", "bc=xmax:neq:0.05,0,0", "bc=ymin:bb", "bc=ymax:bb", "bc=zmin:bb",
                        "bc=zmax:bb"], check=True, cwd=tmp, stdout=subprocess.DEVNULL)
        _, _, levels = load_levels(dump)
    out = {"meta": json.dumps(meta)}
    empty = np.zeros(0, dtype=np.uint64)
    for lv, L in enumerate(levels):
        out[f"codes{lv}"] = L["nodes"]["code"].copy()
        out[f"flags{lv}"] = L["nodes"]["flag"].copy()
        lay = L["layers"]
        out[f"c2f_fine{lv}"] = np.union1d(np.union1d(lay.get((2, 1), empty), lay.get((3, 1), empty)),
                                          np.union1d(lay.get((2, 2), empty), lay.get((3, 2), empty)))
        out[f"f2c_coarse{lv}"] = np.union1d(lay.get((0, 1), empty), lay.get((1, 1), empty))
    np.savez_compressed(a.out, **out)
    print(a.out, [int(out[f"codes{lv}"].size) for lv in range(len(levels))], "nodes per level")


if __name__ == "__main__":
    main()
