"""Immersed-boundary forcing with the reference's four-point kernel and the three-point kernel of
Roma, Peskin and Berger: vertex forces against the oracle's interpolation (FP64, 1e-12), and the
spread force entering the momentum balance exactly (periodic box: the step changes the total
momentum by the sum of the node forces)."""
import numpy as np
import pytest

import zllbm_b200 as zl
from oracle import ib

pytestmark = pytest.mark.gpu

C9 = np.array([(0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, 1), (-1, -1), (1, -1)], dtype=np.float64)
W9 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def _feq(rho, u):
    cu = u @ C9.T
    return W9 * rho[:, None] * (1 + 3 * cu + 4.5 * cu ** 2 - 1.5 * (u ** 2).sum(1)[:, None])


@pytest.mark.parametrize("width", [3, 4])
def test_ib_vertex_forces_and_momentum(width):
    n = 40
    codes = zl.box_codes(2, (0, 0), (n - 1, n - 1))
    from oracle.port import morton_decode
    idx = morton_decode(codes, 2)
    x, y = idx[:, 0].astype(np.float64), idx[:, 1].astype(np.float64)
    u = np.stack([0.02 * np.sin(2 * np.pi * y / n), 0.015 * np.cos(2 * np.pi * x / n)], axis=1)
    rho = 1.0 + 0.001 * np.sin(2 * np.pi * (x + y) / n)
    f = _feq(rho, u)
    nv = 44
    th = np.arange(nv) * 2 * np.pi / nv
    coords = np.stack([20.3 + 7 * np.cos(th), 19.7 + 7 * np.sin(th), np.zeros(nv)], axis=1)
    vel = np.stack([-0.01 * np.sin(th), 0.01 * np.cos(th), np.zeros(nv)], axis=1)
    area = np.full(nv, 2 * np.pi * 7 / nv)
    cfg = zl.SolverConfig(lattice=zl.D2Q9, collision=zl.SRT, storage=zl.STORAGE_F64, viscosity=0.05,
                          bc_kind=(zl.BC_PERIODIC,) * 4 + (0, 0), domain_min=(0, 0, 0), domain_max=(n, n, 0),
                          forcing=1)
    with zl.Context(cfg) as ctx:
        ctx.set_level_box(0, (0, 0, 0), (n, n, 1))  # periodic: the box wraps on both axes
        ctx.set_populations(0, codes, f)
        ctx.ib_set_delta(0, width)
        ctx.ib_set_vertices(0, coords, vel, area)
        before = ctx.conservation(0)
        ctx.step_level(0)
        after = ctx.conservation(0)
        forces, total = ctx.ib_get_forces(0)
    # oracle: node velocities from the populations the step started from
    grid_u = np.zeros((n, n, 3))
    r = f.sum(1)
    grid_u[idx[:, 1], idx[:, 0], :2] = (f @ C9) / r[:, None]
    ref = ib.vertex_forces(lambda jx, jy: grid_u[jy % n, jx % n], coords, vel, 1.0, width)
    np.testing.assert_allclose(forces, ref, rtol=1e-12, atol=1e-15)
    # the step adds sum(node force) dt to the momentum; spreading keeps sum F area / dx
    spread = (forces[:, :2] * area[:, None]).sum(0)
    np.testing.assert_allclose(after[1:3] - before[1:3], spread, rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(total[:2], spread, rtol=1e-12, atol=1e-15)
