"""GPU Smagorinsky LES (tau = tau0 + tau_sgs, Cs configurable) against the oracle restatement."""
import numpy as np
import pytest

from fixtures import grid_order

pytestmark = pytest.mark.gpu
zl = pytest.importorskip("zllbm_b200")


def run_both(port, cfg, f_grid, steps, storage, cs):
    from oracle.port import morton_decode  # noqa: F401
    dims = cfg.dims
    codes = zl.box_codes(dims, [1] * dims, list(cfg.n[:dims]))
    lin = grid_order(codes, dims, cfg.n)
    f = np.ascontiguousarray(f_grid.reshape(-1, cfg.q))
    f0 = f[lin].copy()
    cfg.les, cfg.les_cs = 1, cs
    port.run(cfg, f, f.copy(), steps)
    scfg = zl.SolverConfig(lattice=zl.D2Q9 if dims == 2 else zl.D3Q19, collision=cfg.collision, storage=storage,
                           viscosity=cfg.nu, bc_kind=tuple(cfg.bc_kind), bc_velocity=tuple(cfg.bc_vel),
                           domain_min=(1, 1, 1 if dims == 3 else 0),
                           domain_max=tuple(list(cfg.n[:dims]) + [0] * (3 - dims)), les=1, les_cs=cs)
    with zl.Context(scfg) as ctx:
        ctx.set_level_nodes(0, codes)
        ctx.set_populations(0, codes, f0)
        ctx.advance(steps)
        got = ctx.get_populations(0, codes)
    return got, f[lin]


@pytest.mark.parametrize("coll", [0, 1])
@pytest.mark.parametrize("storage,tol", [(zl.STORAGE_F64, 0.0), (zl.STORAGE_F32, 1e-5)])
def test_les_tgv(port, coll, storage, tol):
    from oracle.port import BC_PERIODIC, LevelConfig, tgv_init
    cfg = LevelConfig(dims=3, n=(13, 13, 13), collision=coll, nu=0.001, bc_kind=(BC_PERIODIC,) * 6)
    f = tgv_init(cfg, 0.08, port)
    got, ref = run_both(port, cfg, f, 25, storage, 0.1)
    err = np.abs(got - ref) / np.abs(ref)
    assert err.max() <= tol, err.max()


@pytest.mark.parametrize("coll", [0, 1])
def test_les_cavity_fp64(port, coll):
    from oracle.port import BC_BOUNCE_BACK, LevelConfig
    z3 = (0.0, 0.0, 0.0)
    cfg = LevelConfig(dims=2, n=(20, 20), collision=coll, nu=0.002, bc_kind=(BC_BOUNCE_BACK,) * 4 + (0, 0),
                      bc_vel=(z3, z3, z3, (0.1, 0, 0), z3, z3))
    f = np.tile(port.feq(2, 1.0, [0.0, 0.0]), (400, 1)).reshape(20, 20, 9)
    got, ref = run_both(port, cfg, f, 60, zl.STORAGE_F64, 0.16)
    assert np.array_equal(got, ref), np.abs(got - ref).max()
