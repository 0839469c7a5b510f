"""GPU parity: the CUDA path through the C ABI against the reference's own outputs and the oracle."""
import os

import numpy as np
import pytest

from fixtures import GOLDEN, grid_order, level_config, lbm_fixture_names, load_lbm, solver_config

pytestmark = pytest.mark.gpu

zl = pytest.importorskip("zllbm_b200")


def run_gpu(meta, codes, f0, storage, steps=None):
    cfg = solver_config(meta, storage)
    with zl.Context(cfg) as ctx:
        ctx.set_level_nodes(0, codes)
        ctx.set_populations(0, codes, f0)
        ctx.advance(meta["steps"] if steps is None else steps)
        f = ctx.get_populations(0, codes)
        rho, u = ctx.get_macros(0, codes)
    return f, rho, u


def velocity(meta, f):
    from oracle.port import LATTICE_C
    c = np.array(LATTICE_C[meta["dims"]], dtype=np.float64)
    rho = f.sum(1)
    return (f @ c) / rho[:, None]


@pytest.mark.parametrize("name", lbm_fixture_names())
def test_fp64_bit_exact_against_reference(name):
    """FP64 storage reproduces the reference's doubles bit for bit (tolerance: 0 ulp)."""
    meta, codes, f0, f1 = load_lbm(name)
    f, _, _ = run_gpu(meta, codes, f0, zl.STORAGE_F64)
    assert np.array_equal(f, f1), f"max |diff| = {np.abs(f - f1).max():.3e}"


@pytest.mark.parametrize("name", lbm_fixture_names())
def test_fp32_against_reference(name):
    """FP32 deviation storage: populations within 1e-5 relative of the reference's FP64."""
    meta, codes, f0, f1 = load_lbm(name)
    f, _, _ = run_gpu(meta, codes, f0, zl.STORAGE_F32)
    rel = np.abs(f - f1) / np.abs(f1)
    assert rel.max() <= 1e-5, rel.max()


@pytest.mark.parametrize("storage,tol", [(zl.STORAGE_F16, 5e-3), (zl.STORAGE_BF16, 5e-2)])
@pytest.mark.parametrize("name", ["tgv3d_mrt", "tgv3d_srt", "tgv2d_mrt"])
def test_reduced_storage_velocity(name, storage, tol):
    """FP16 / BF16 deviation storage: relative L2 velocity error vs the reference (stated tolerance)."""
    meta, codes, f0, f1 = load_lbm(name)
    _, _, u = run_gpu(meta, codes, f0, storage)
    u_ref = velocity(meta, f1)
    err = np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref)
    assert err <= tol, err


def test_macros_match_reference_output_rule():
    meta, codes, f0, f1 = load_lbm("cavity2d_srt")
    f, rho, u = run_gpu(meta, codes, f0, zl.STORAGE_F64)
    assert np.array_equal(rho, f1.sum(1)) or np.allclose(rho, f1.sum(1), rtol=1e-15, atol=0)
    assert np.allclose(u, velocity(meta, f1), rtol=0, atol=1e-15)


@pytest.mark.parametrize("case", ["tgv3d", "cavity2d", "channel3d"])
def test_fp64_bit_exact_against_oracle_larger(case, port):
    """Sizes beyond the committed fixtures, against the oracle restatement (itself pinned above)."""
    from oracle.port import BC_BOUNCE_BACK, BC_NONEQ, BC_PERIODIC, MRT, SRT, LevelConfig, tgv_init
    z3 = (0.0, 0.0, 0.0)
    if case == "tgv3d":
        cfg = LevelConfig(dims=3, n=(33, 33, 33), collision=MRT, nu=0.05 / 3, bc_kind=(BC_PERIODIC,) * 6)
        f = tgv_init(cfg, 0.05, port)
        steps = 60
    elif case == "cavity2d":
        cfg = LevelConfig(dims=2, n=(64, 64), collision=SRT, nu=0.064, bc_kind=(BC_BOUNCE_BACK,) * 4 + (0, 0),
                          bc_vel=(z3, z3, z3, (0.1, 0, 0), z3, z3))
        f = np.tile(port.feq(2, 1.0, [0.0, 0.0]), (64 * 64, 1)).reshape(64, 64, 9)
        steps = 500
    else:
        cfg = LevelConfig(dims=3, n=(24, 12, 10), collision=MRT, nu=0.02,
                          bc_kind=(BC_NONEQ, BC_NONEQ, BC_BOUNCE_BACK, BC_BOUNCE_BACK, BC_BOUNCE_BACK, BC_BOUNCE_BACK),
                          bc_vel=((0.04, 0, 0), (0.04, 0, 0), z3, z3, z3, z3))
        f = np.tile(port.feq(3, 1.0, [0.0, 0.0, 0.0]), (24 * 12 * 10, 1)).reshape(10, 12, 24, 19)
        steps = 80
    meta = dict(dims=cfg.dims, n=list(cfg.n), collision=cfg.collision, nu=cfg.nu, rho0=cfg.rho0,
                bc_kind=list(cfg.bc_kind), bc_vel=[list(v) for v in cfg.bc_vel], steps=steps)
    f = np.ascontiguousarray(f.reshape(-1, cfg.q))
    codes = zl.box_codes(cfg.dims, [1] * cfg.dims, list(cfg.n[: cfg.dims]))
    lin = grid_order(codes, cfg.dims, cfg.n)
    f_nodes = f[lin].copy()
    port.run(cfg, f, f.copy(), steps)
    got, _, _ = run_gpu(meta, codes, f_nodes, zl.STORAGE_F64)
    assert np.array_equal(got, f[lin]), np.abs(got - f[lin]).max()


@pytest.mark.parametrize("dims", [2, 3])
def test_device_morton_neighbors_bit_exact(dims):
    z = np.load(os.path.join(GOLDEN, f"morton_{dims}d.npz"))
    assert np.array_equal(zl.morton_neighbors(dims, z["codes"]), z["neighbors"])


@pytest.mark.parametrize("lattice", [2, 3])
def test_device_upstream_index_matches_hash_lookup(lattice):
    from oracle.port import upstream_lookup
    dims = 2 if lattice == zl.D2Q9 else 3
    rng = np.random.default_rng(11 + dims)
    hi = [20, 17, 9][:dims]
    all_codes = zl.box_codes(dims, [1] * dims, hi)
    keep = rng.random(all_codes.size) < 0.6
    codes = rng.permutation(all_codes[keep])
    assert np.array_equal(zl.upstream_index(lattice, codes), upstream_lookup(codes, dims))


def test_conservation_fp64_periodic(port):
    meta, codes, f0, f1 = load_lbm("tgv3d_mrt")
    cfg = solver_config(meta, zl.STORAGE_F64)
    with zl.Context(cfg) as ctx:
        ctx.set_level_nodes(0, codes)
        ctx.set_populations(0, codes, f0)
        m0 = ctx.conservation(0)
        ctx.advance(200)
        m1 = ctx.conservation(0)
    assert abs(m1[0] - m0[0]) / m0[0] < 1e-13
    assert np.all(np.abs(m1[1:]) < 1e-12)


def test_error_paths():
    meta, codes, f0, f1 = load_lbm("cavity2d_srt")
    cfg = solver_config(meta, zl.STORAGE_F32)
    with zl.Context(cfg) as ctx:
        with pytest.raises(zl.ZlError) as e:
            ctx.step_level(0)
        assert e.value.code == -6
        ctx.set_level_nodes(0, codes)
        bad = zl.box_codes(2, [30, 30], [31, 31])
        with pytest.raises(zl.ZlError) as e:
            ctx.set_populations(0, bad, np.zeros((bad.size, 9)))
        assert e.value.code == -2
        with pytest.raises(zl.ZlError) as e:
            ctx.set_level_nodes(0, zl.box_codes(2, [1, 1], [40, 40]))
        assert e.value.code == -2


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [0, 2])
def test_exchange_without_codes_uses_the_level_order(storage):
    """Node exchanges with codes = NULL cover the level's own node list in the order handed to
    zl_set_level_nodes (kept on the device): same results as passing those codes, and a count
    other than the level's is refused."""
    import zllbm_b200 as zl
    meta, codes, f0, _ = load_lbm("box3d_mixed")
    order = np.random.default_rng(3).permutation(codes.size)
    shuffled = codes[order]
    with zl.Context(solver_config(meta, storage)) as ctx:
        ctx.set_level_nodes(0, shuffled)
        ctx.set_populations(0, None, f0[order])
        ctx.advance(3)
        a = ctx.get_populations(0, shuffled)
        b = ctx.get_populations(0, None, codes.size)
        assert np.array_equal(a, b)
        rho_a, u_a = ctx.get_macros(0, shuffled)
        rho_b, u_b = ctx.get_macros(0, None, codes.size)
        assert np.array_equal(rho_a, rho_b) and np.array_equal(u_a, u_b)
        with pytest.raises(zl.ZlError) as e:
            ctx.get_populations(0, None, codes.size - 1)
        assert e.value.code == -1  # ZL_EINVAL
    with zl.Context(solver_config(meta, storage)) as ctx:
        ctx.set_level_nodes(0, shuffled)
        ctx.set_populations(0, shuffled, f0[order])
        ctx.advance(3)
        assert np.array_equal(ctx.get_populations(0, shuffled), a)
