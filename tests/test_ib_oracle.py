"""The oracle's immersed-boundary interpolation pinned to the reference: one step of the reference's
direct forcing (a circle in 2D, a sphere in 3D, four-point kernel) from a Taylor-Green velocity
field (tests/golden/ibpin_*.npz, ``python tests/golden/make_golden.py ibpin``).  The vertex forces
the reference stores after the step come from the first pass, which reads the initial
populations, so F = 2 (U_b - sum delta u) restated on those populations must give them to
rounding; spread into node forces and fed to the oracle's forced step, they must give the
reference's populations after the step."""
import json
import os

import numpy as np
import pytest

from oracle import ib
from oracle.port import LATTICE_C, morton_decode

HERE = os.path.dirname(os.path.abspath(__file__))


def velocities(codes, f, dims):
    """Node velocity from the populations, keyed by level indices (the reference's macro of a node
    whose immersed-boundary force was reset, no other force)."""
    c = np.array(LATTICE_C[dims], dtype=np.float64)
    u = (f @ c) / f.sum(1)[:, None]
    out = np.zeros((len(codes), 3))
    out[:, :dims] = u
    return {tuple(i): v for i, v in zip(morton_decode(codes, dims).tolist(), out)}


@pytest.mark.parametrize("name", ["ib2d", "ib3d"])
def test_vertex_forces_match_reference_first_pass(name):
    z = np.load(os.path.join(HERE, "golden", f"ibpin_{name}.npz"))
    meta = json.loads(str(z["meta"]))
    dims = meta["dims"]
    before, after = z["vertices_before"], z["vertices_after"]
    assert np.array_equal(before[:, :7], after[:, :7])  # vertices do not move
    u = velocities(z["codes0"], z["f_before0"], dims)
    ref = after[:, 7:10]
    assert np.abs(ref[:, :dims]).max() > 1e-3  # the field is not uniform around the body
    got = ib.vertex_forces(lambda *j: u[j], before[:, 0:3], before[:, 3:6], 1.0, 4, dims)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("name", ["ib2d", "ib3d"])
def test_one_forced_step_matches_reference(name, port):
    """Interpolation, spreading and the forced collision together: the oracle's node forces fed to
    the restated step reproduce the reference's populations after the step."""
    from fixtures import grid_order
    from oracle.port import BC_PERIODIC, SRT, LevelConfig
    z = np.load(os.path.join(HERE, "golden", f"ibpin_{name}.npz"))
    meta = json.loads(str(z["meta"]))
    dims = meta["dims"]
    n = [v + 1 for v in meta["n"]]  # stored nodes: both periodic planes
    nn = int(np.prod(n))
    lin = grid_order(z["codes0"], dims, n)
    q = z["f_before0"].shape[1]
    f = np.empty((nn, q))
    f[lin] = z["f_before0"]
    v = z["vertices_before"]
    u = velocities(z["codes0"], z["f_before0"], dims)
    forces = ib.vertex_forces(lambda *j: u[j], v[:, 0:3], v[:, 3:6], 1.0, 4, dims)
    node_force = np.zeros((nn, 3))

    def add(j, share):
        k = (j[0] - 1) + n[0] * (j[1] - 1) + (n[0] * n[1] * (j[2] - 1) if dims == 3 else 0)
        node_force[k] += share

    ib.spread(forces, v[:, 0:3], v[:, 6], 1.0, 1.0, 4, dims, add)
    assert np.abs(node_force).max() > 1e-3
    cfg = LevelConfig(dims=dims, n=tuple(n), collision=SRT, nu=meta["nu"],
                      bc_kind=(BC_PERIODIC,) * (2 * dims) + (0,) * (6 - 2 * dims), node_force=node_force)
    port.run(cfg, f, f.copy(), 1)
    # node forces sum the vertex shares in another order than the reference's unordered_map walk:
    # populations agree to an ulp (about 3e-17 here), not bit for bit
    np.testing.assert_allclose(f[lin], z["f_after0"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("name", ["amr_ib2d_l0", "amr_ib2d_l1", "ibpin_ib2d"])
def test_reference_circle_vertex_count_and_arc(name):
    """The reference's circle (geometry_default_shape_2d.cpp:34) has floor(2 pi r / dx_l) + 1
    vertices on its level, each with arc 2 pi r / count (UpdateShape), placed on the circle."""
    import math
    z = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    meta = json.loads(str(z["meta"]))
    r = float(meta["ib"].split(":")[1].split(",")[2])
    dx = 1.0 / (1 << meta["levels"])
    v = z["vertices_before"]
    assert len(v) == math.floor(2 * math.pi * r / dx) + 1
    np.testing.assert_allclose(v[:, 6], 2 * math.pi * r / len(v), rtol=1e-12)
    rad = np.hypot(v[:, 0] - v[:, 0].mean(), v[:, 1] - v[:, 1].mean())
    np.testing.assert_allclose(rad, r, rtol=1e-9)
