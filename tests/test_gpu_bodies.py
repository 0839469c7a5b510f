"""The multi-level flow drivers (flow past a cube: D3Q19 SRT + Smagorinsky + immersed boundary on
three levels; flow past a cylinder: D2Q9 MRT + immersed boundary on three levels) on small grids
refined by the reference's own grid builder (tests/golden/topo_*_small.npz, written by
``python tests/golden/make_golden.py topo``).

Each runs a few coarse steps as batched launches replayed from a CUDA graph and again launch by
launch; the body forces and level masses agree (FP32 storage, node forces spread with atomics, so
to a relative 1e-4) and stay finite.  Without a GPU: the fixtures' interface layers lie in their
levels, and every stencil node of the drivers' body vertices exists on the finest level.
"""
import itertools
import json
import math
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
TOPOS = ("topo_cube_small", "topo_cylinder_small")


def load_topo(name):
    z = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    return json.loads(str(z["meta"])), z


def body_vertices(meta):
    from zllbm_b200.cube_flow import cube_vertices
    from zllbm_b200.cylinder_flow import VERTICES
    h = 1.0 / (1 << meta["levels"])
    if "cube" in meta:
        cx, cy, cz, edge = (float(v) for v in meta["cube"].split(","))
        return cube_vertices((cx, cy, cz), edge, h)[0]
    cx, cy, r = (float(v) for v in meta["circle"].split(","))
    t = 2.0 * math.pi * np.arange(VERTICES) / VERTICES
    return np.stack([cx + r * np.cos(t), cy + r * np.sin(t), np.zeros(VERTICES)], axis=1)


@pytest.mark.parametrize("name", TOPOS)
def test_topology_fixture_layers_are_consistent(name):
    meta, z = load_topo(name)
    for lv in range(meta["levels"] + 1):
        codes = z[f"codes{lv}"]
        assert codes.size > 0 and z[f"flags{lv}"].size == codes.size
        assert np.all(np.diff(codes.astype(np.uint64)) > 0)  # sorted, distinct
    for lv in range(1, meta["levels"] + 1):
        assert z[f"c2f_fine{lv}"].size > 0 and z[f"f2c_coarse{lv - 1}"].size > 0
        assert np.isin(z[f"c2f_fine{lv}"], z[f"codes{lv}"]).all()
        assert np.isin(z[f"f2c_coarse{lv - 1}"], z[f"codes{lv - 1}"]).all()


@pytest.mark.parametrize("name", TOPOS)
def test_every_body_stencil_node_is_on_the_finest_level(name):
    """The drivers put the body's vertices on the finest level; the four-point stencil of each
    (first node (uint32)(x / dx + 1e-6) - 1 per axis) must find all its nodes there."""
    from oracle.port import morton_decode
    meta, z = load_topo(name)
    dims, levels = meta["dims"], meta["levels"]
    have = set(map(tuple, morton_decode(z[f"codes{levels}"], dims).tolist()))
    dx = 1.0 / (1 << levels)
    for p in body_vertices(meta):
        first = [int(p[a] / dx + 1e-6) - 1 for a in range(dims)]
        for o in itertools.product(range(4), repeat=dims):
            assert tuple(first[a] + o[a] for a in range(dims)) in have


def quiet(*_):
    pass


def check_pair(fast, plain):
    assert fast["finite"] and plain["finite"]
    assert fast["nodes_per_level"] == plain["nodes_per_level"]
    assert all(n > 0 for n in fast["nodes_per_level"])
    key = "cube_force_total" if "cube_force_total" in fast else "cylinder_force_total_fp64"
    a, b = np.asarray(fast[key]), np.asarray(plain[key])
    scale = float(np.abs(b).max())
    assert scale > 0.0
    np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-4 * scale)
    if "mass_per_level" in fast:
        np.testing.assert_allclose(fast["mass_per_level"], plain["mass_per_level"], rtol=1e-5)


@pytest.mark.gpu
def test_cube_flow_graph_matches_plain():
    from zllbm_b200 import cube_flow
    topo = os.path.join(HERE, "golden", "topo_cube_small.npz")
    fast = cube_flow.run(topo, steps=6, warmup=2, graph=True, batching=True, log=quiet)
    plain = cube_flow.run(topo, steps=6, warmup=2, graph=False, batching=False, streams=False, log=quiet)
    check_pair(fast, plain)


@pytest.mark.gpu
def test_cylinder_flow_graph_matches_plain():
    from zllbm_b200 import cylinder_flow
    topo = os.path.join(HERE, "golden", "topo_cylinder_small.npz")
    fast = cylinder_flow.run(topo, steps=6, warmup=2, graph=True, batching=True, log=quiet)
    plain = cylinder_flow.run(topo, steps=6, warmup=2, graph=False, batching=False, streams=False, log=quiet)
    check_pair(fast, plain)


def test_cube_surface_vertices():
    """Host geometry of the cube-flow driver: every grid point of the six faces once, on the
    surface, with areas summing to the cube's surface."""
    from zllbm_b200.cube_flow import cube_vertices
    edge, h, centre = 4.0, 0.25, np.array([16.0, 16.0, 16.0])
    xyz, area = cube_vertices(tuple(centre), edge, h)
    m = int(edge / h)
    assert len(xyz) == (m + 1) ** 3 - (m - 1) ** 3  # surface points of an (m+1)^3 lattice cube
    assert len(np.unique(np.round(xyz / h).astype(np.int64), axis=0)) == len(xyz)
    d = np.abs(xyz - centre)
    assert np.all(np.isclose(d.max(1), edge / 2))  # on the surface
    assert area.sum() == pytest.approx(6 * edge * edge, rel=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("flow", ["cube", "cylinder"])
def test_level_streams_are_bit_exact(flow):
    """The sub-cycled order on per-level streams (immersed-boundary passes beside the transfers of
    their level) and on one stream give the same vertex forces and level masses bit for bit."""
    from zllbm_b200 import cube_flow, cylinder_flow
    mod = cube_flow if flow == "cube" else cylinder_flow
    topo = os.path.join(HERE, "golden", f"topo_{flow}_small.npz")
    a = mod.run(topo, steps=6, warmup=2, graph=True, batching=False, streams=True, log=quiet)
    b = mod.run(topo, steps=6, warmup=2, graph=False, batching=False, streams=False, log=quiet)
    key = "cube_force_total" if flow == "cube" else "cylinder_force_total_fp64"
    assert a[key] == b[key]
    if "mass_per_level" in a:
        assert a["mass_per_level"] == b["mass_per_level"]
