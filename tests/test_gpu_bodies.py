"""The multi-level flow drivers (flow past a cube: D3Q19 SRT + Smagorinsky + immersed boundary on
three levels; flow past a cylinder: D2Q9 MRT + immersed boundary on three levels) on small grids
refined by the reference's own grid builder (tests/golden/topo_*_small.npz, written by
``python tests/golden/make_golden.py topo``).

Each runs a few coarse steps as batched launches replayed from a CUDA graph and again launch by
launch; the body forces and level masses agree (FP32 storage, node forces spread with atomics, so
to a relative 1e-4) and stay finite.
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


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
    plain = cube_flow.run(topo, steps=6, warmup=2, graph=False, batching=False, log=quiet)
    check_pair(fast, plain)


@pytest.mark.gpu
def test_cylinder_flow_graph_matches_plain():
    from zllbm_b200 import cylinder_flow
    topo = os.path.join(HERE, "golden", "topo_cylinder_small.npz")
    fast = cylinder_flow.run(topo, steps=6, warmup=2, graph=True, batching=True, log=quiet)
    plain = cylinder_flow.run(topo, steps=6, warmup=2, graph=False, batching=False, log=quiet)
    check_pair(fast, plain)
