"""The packed topology format (zllbm_b200/topology_pack.py) keeps the reference-built node sets
and interface layers exactly: round trips of the committed small grids built by the reference's
grid builder, and the level sizes of the packed full-size grids the flow drivers and the
benchmark use."""
import json
import os

import numpy as np
import pytest

from fixtures import GOLDEN

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "zllbm_b200")


@pytest.mark.parametrize("name", ["topo_cube_small", "topo_cylinder_small"])
def test_pack_round_trip(name, tmp_path):
    from zllbm_b200 import topology_pack as tp
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    src = {k: z[k] for k in z.files}
    path = tmp_path / "packed.npz"
    np.savez_compressed(path, **tp.pack(src))
    back = tp.load_topology(str(path))
    assert json.loads(str(back["meta"])) == json.loads(str(src["meta"]))
    lv = 0
    while f"codes{lv}" in src:
        codes = src[f"codes{lv}"]
        assert np.array_equal(back[f"codes{lv}"], np.sort(codes))
        for key in ("c2f_fine", "f2c_coarse"):
            assert np.array_equal(back[f"{key}{lv}"], np.sort(src[f"{key}{lv}"]))
        ghost = np.sort(codes[(src[f"flags{lv}"] & 4) != 0])
        assert np.array_equal(back[f"codes{lv}"][(back[f"flags{lv}"] & 4) != 0], ghost)
        lv += 1
    assert lv >= 3


@pytest.mark.parametrize("name,nodes", [
    ("cube_256x128x128_l2", [4237533, 347391, 749331]),
    ("cylinder_1024x512_l3", [524675, 4469, 4486, 5159]),
])
def test_packed_full_size_topologies(name, nodes):
    from zllbm_b200 import topology_pack as tp
    z = np.load(os.path.join(PKG, "topologies", f"{name}.npz"))
    meta = json.loads(str(z["meta"]))
    assert meta["levels"] == len(nodes) - 1
    dims = meta["dims"]
    for lv, n in enumerate(nodes):
        box = z[f"box{lv}"]
        assert n <= int(np.prod(box[dims:]))
    if name.startswith("cylinder"):  # small enough to unpack here
        back = tp.load(os.path.join(PKG, "topologies", f"{name}.npz"))
        assert [back[f"codes{lv}"].size for lv in range(len(nodes))] == nodes
