"""Node sets and interface layers of a multi-level grid refined around a body, generated by the
reference's own grid builder (refinement around a GeometryInfoOrigin cube or circle,
AmrManager::SetupMesh) through the oracle harness, and saved as the input of
``python -m zllbm_b200.cube_flow`` (3D cube) or ``python -m zllbm_b200.cylinder_flow`` (2D circle).

    python oracle/make_body_topology.py OUT.npz [--n 256,128,128] [--levels 2] [--cube 80,64,64,16]
                                                [--ext 6] [--inner 16]
    python oracle/make_body_topology.py OUT.npz --n 1024,512 --levels 3 --circle 256,256,2.5 --ext 6 --inner 8

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
    ap.add_argument("--circle", default=None, help="cx,cy,r: a 2D grid refined around a circle")
    ap.add_argument("--ext", default="6")
    ap.add_argument("--inner", default="16")
    a = ap.parse_args(argv)
    if not os.path.exists(REF_RUN):
        subprocess.run(["make", "-C", HERE, "ref"], check=True)
    dims = 2 if a.circle else 3
    meta = {"dims": dims, "n": [int(v) for v in a.n.split(",")], "levels": a.levels, "ext": a.ext, "inner": a.inner}
    if a.circle:
        meta["circle"] = a.circle
        geo = f"geo=circle:{a.circle}"
        bcs = ["bc=xmin:neq:0.04,0", "bc=xmax:neq:0.04,0", "bc=ymin:bb", "bc=ymax:bb"]
    else:
        meta["cube"] = a.cube
        geo = f"geo=cube:{a.cube}"
        bcs = ["bc=xmin:neq:0.05,0,0", "bc=xmax:neq:0.05,0,0", "bc=ymin:bb", "bc=ymax:bb", "bc=zmin:bb", "bc=zmax:bb"]
    with tempfile.TemporaryDirectory() as tmp:
        dump = os.path.join(tmp, "l0.bin")
        subprocess.run([REF_RUN, f"dims={dims}", f"n={a.n}", f"levels={a.levels}", geo, f"ext={a.ext}",
                        f"inner={a.inner}", "coll=srt", "nu=0.01", "steps=0", f"lout0={dump}"] + bcs,
                       check=True, cwd=tmp, stdout=subprocess.DEVNULL)
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
