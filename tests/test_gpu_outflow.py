"""Convective outflow faces (no counterpart in the reference) against the C restatement:
FP64 bit for bit, FP32 within 1e-5, on channels with a non-equilibrium inflow."""
import numpy as np
import pytest

import zllbm_b200 as zl
from fixtures import grid_order
from test_gpu_parity import run_gpu

pytestmark = pytest.mark.gpu


def _channel(dims, coll, conv_face="xmax", inflow_face="xmin"):
    from oracle.port import BC_BOUNCE_BACK, BC_CONVECTIVE, BC_NONEQ, BC_PERIODIC, FACES, LevelConfig
    z3 = (0.0, 0.0, 0.0)
    kinds = [BC_BOUNCE_BACK] * 6
    vels = [z3] * 6
    kinds[FACES.index(inflow_face)] = BC_NONEQ
    vels[FACES.index(inflow_face)] = (0.05, 0.0, 0.0)
    kinds[FACES.index(conv_face)] = BC_CONVECTIVE
    vels[FACES.index(conv_face)] = (0.05, 0.0, 0.0)
    if dims == 3:
        kinds[4] = kinds[5] = BC_PERIODIC
    else:
        kinds[4] = kinds[5] = 0
    n = (40, 16) if dims == 2 else (24, 12, 10)
    return LevelConfig(dims=dims, n=n, collision=coll, nu=0.02, bc_kind=tuple(kinds), bc_vel=tuple(vels))


@pytest.mark.parametrize("dims,coll", [(2, 0), (2, 1), (3, 0), (3, 1)])
def test_convective_outflow_fp64_bit_exact(dims, coll, port):
    cfg = _channel(dims, coll)
    nn = int(np.prod(cfg.n[:dims]))
    f = np.tile(port.feq(dims, 1.0, [0.0] * dims), (nn, 1))
    steps = 150
    meta = dict(dims=dims, n=list(cfg.n), collision=coll, nu=cfg.nu, rho0=cfg.rho0, bc_kind=list(cfg.bc_kind),
                bc_vel=[list(v) for v in cfg.bc_vel], steps=steps)
    codes = zl.box_codes(dims, [1] * dims, list(cfg.n[:dims]))
    lin = grid_order(codes, dims, cfg.n)
    f_nodes = f[lin].copy()
    port.run(cfg, f, f.copy(), steps)
    got, _, _ = run_gpu(meta, codes, f_nodes, zl.STORAGE_F64)
    assert np.array_equal(got, f[lin]), np.abs(got - f[lin]).max()
    got32, _, _ = run_gpu(meta, codes, f_nodes, zl.STORAGE_F32)
    assert np.abs(got32 - f[lin]).max() <= 1e-5 * np.abs(f).max()


def test_convective_outflow_on_a_min_face(port):
    cfg = _channel(2, 0, conv_face="xmin", inflow_face="xmax")
    cfg.bc_vel = tuple((-0.05, 0.0, 0.0) if k in (3, 4) else v for k, v in zip(cfg.bc_kind, cfg.bc_vel))
    nn = int(np.prod(cfg.n[:2]))
    f = np.tile(port.feq(2, 1.0, [0.0, 0.0]), (nn, 1))
    meta = dict(dims=2, n=list(cfg.n), collision=0, nu=cfg.nu, rho0=cfg.rho0, bc_kind=list(cfg.bc_kind),
                bc_vel=[list(v) for v in cfg.bc_vel], steps=120)
    codes = zl.box_codes(2, [1, 1], list(cfg.n[:2]))
    lin = grid_order(codes, 2, cfg.n)
    f_nodes = f[lin].copy()
    port.run(cfg, f, f.copy(), 120)
    got, _, _ = run_gpu(meta, codes, f_nodes, zl.STORAGE_F64)
    assert np.array_equal(got, f[lin])


def test_convective_outflow_needs_a_speed():
    cfg = zl.SolverConfig(lattice=zl.D2Q9, bc_kind=(1, zl.BC_CONVECTIVE_OUTFLOW, 1, 1, 0, 0),
                          domain_min=(1, 1, 0), domain_max=(8, 8, 0))
    with pytest.raises(zl.ZlError):
        zl.Context(cfg)
