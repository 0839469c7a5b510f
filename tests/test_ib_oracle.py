"""The oracle's immersed-boundary interpolation pinned to the reference: one step of the reference's
direct forcing (a circle in 2D, a sphere in 3D, four-point kernel) from a Taylor-Green velocity
field (tests/golden/ibpin_*.npz, ``python tests/golden/make_golden.py ibpin``).  The vertex forces
the reference stores after the step come from the first pass, which reads the initial
populations, so F = 2 (U_b - sum delta u) restated on those populations must give them to
rounding."""
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
