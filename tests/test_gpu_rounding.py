"""Stochastic rounding of FP16 / BF16 populations (zl_config.storage_rounding = ZL_ROUND_STOCHASTIC):
the one-node, two-nodes-per-thread and one-warp-per-row step kernels stay within the reduced-
storage tolerances of the oracle; results are deterministic (graph replay equals launch by launch);
and the rounding is unbiased: from a uniform flow on the 16-bit grid, the box mean of every stored
population after one step equals the exact post-collision value to 0.05 ulp."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = (129, 9, 8)  # 128-node periodic rows: every kernel applies
SHAPES = {"scalar": (128, 1), "pair": (-64, 1), "row": (1 << 20, 4)}


def _meta(coll):
    from oracle.port import BC_PERIODIC
    return dict(dims=3, n=list(N), collision=coll, nu=0.05 / 3, rho0=1.0, bc_kind=[BC_PERIODIC] * 6,
                bc_vel=[[0.0, 0.0, 0.0]] * 6)


def _config(meta, storage, rounding):
    from fixtures import solver_config
    cfg = solver_config(meta, storage)
    cfg.storage_rounding = rounding
    return cfg


@pytest.mark.parametrize("storage,tol", [(2, 5e-3), (3, 5e-2)])
@pytest.mark.parametrize("kernel", sorted(SHAPES))
def test_stochastic_rounding_against_oracle(kernel, storage, tol, port):
    import zllbm_b200 as zl
    from fixtures import grid_order
    from oracle.port import MRT, LevelConfig, tgv_init
    from test_gpu_parity import velocity
    meta = _meta(MRT)
    cfg = LevelConfig(dims=3, n=N, collision=MRT, nu=meta["nu"], bc_kind=tuple(meta["bc_kind"]))
    steps = 13
    f = np.ascontiguousarray(tgv_init(cfg, 0.05, port).reshape(-1, cfg.q))
    codes = zl.box_codes(3, [1, 1, 1], list(N))
    lin = grid_order(codes, 3, N)
    f0 = f[lin].copy()
    port.run(cfg, f, f.copy(), steps)
    f1 = f[lin]
    out = {}
    for rounding in (zl.ROUND_NEAREST, zl.ROUND_STOCHASTIC):
        with zl.Context(_config(meta, storage, rounding)) as ctx:
            ctx.set_level_nodes(0, codes)
            ctx.set_populations(0, codes, f0)
            ctx.set_block(0, *SHAPES[kernel])
            ctx.advance(steps)
            out[rounding] = ctx.get_populations(0, codes)
    ue = velocity(meta, f1)
    ug = velocity(meta, out[zl.ROUND_STOCHASTIC])
    assert np.linalg.norm(ug - ue) / np.linalg.norm(ue) <= tol
    assert not np.array_equal(out[zl.ROUND_STOCHASTIC], out[zl.ROUND_NEAREST])


@pytest.mark.parametrize("storage", [2, 3])
def test_stochastic_rounding_is_deterministic(storage, port):
    """The random bits come from per-level step seeds in device memory and the node / lane index:
    two runs, one replaying a captured graph and one stepping launch by launch, agree bit for bit."""
    import zllbm_b200 as zl
    from oracle.port import MRT, LevelConfig, tgv_init
    from fixtures import grid_order
    meta = _meta(MRT)
    cfg = LevelConfig(dims=3, n=N, collision=MRT, nu=meta["nu"], bc_kind=tuple(meta["bc_kind"]))
    codes = zl.box_codes(3, [1, 1, 1], list(N))
    f0 = np.ascontiguousarray(tgv_init(cfg, 0.05, port).reshape(-1, cfg.q)[grid_order(codes, 3, N)])
    res = []
    for graph in (False, True):
        with zl.Context(_config(meta, storage, zl.ROUND_STOCHASTIC)) as ctx:
            ctx.set_level_nodes(0, codes)
            ctx.set_populations(0, codes, f0)
            ctx.set_block(0, *SHAPES["row"])
            ctx.set_graph(graph)
            if graph:
                ctx.advance(10)
            else:
                for _ in range(10):
                    ctx.step_level(0)
            res.append(ctx.get_populations(0, codes))
    assert np.array_equal(res[0], res[1])


def _representable(dev_scaled, storage):
    """Scaled deviations rounded to the nearest FP16 / BF16 value (numpy has no bfloat16: the FP32
    bit pattern rounded to nearest-even on its upper 16 bits)."""
    if storage == 2:
        return dev_scaled.astype(np.float16).astype(np.float64)
    b = dev_scaled.astype(np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16 << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def _ulp(x_scaled, storage):
    if storage == 2:
        return np.spacing(np.abs(x_scaled).astype(np.float16)).astype(np.float64)
    e = np.floor(np.log2(np.abs(x_scaled)))
    return np.exp2(e - 7)


@pytest.mark.parametrize("storage", [2, 3])
@pytest.mark.parametrize("kernel", sorted(SHAPES))
def test_stochastic_rounding_is_unbiased(kernel, storage, port):
    """One step of a uniform flow whose populations are exactly representable in 16 bits: every
    node collides to the same FP32 values, which are not representable.  Round to nearest stores
    the same neighbour everywhere; stochastic rounding picks either neighbour with the right odds,
    so the box mean of each population lands on the exact post-collision value (the oracle's, in
    FP64) to 0.05 ulp (about 9,000 nodes; a biased choice would miss by up to 1 ulp)."""
    import zllbm_b200 as zl
    from oracle.port import MRT, LevelConfig
    meta = _meta(MRT)
    scale = 8192.0
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
    feq = np.asarray(port.feq(3, 1.0, (0.0123456789, -0.00731, 0.00219)))
    f_exact16 = w + _representable((feq - w) * scale, storage) / scale
    codes = zl.box_codes(3, [1, 1, 1], list(N))
    f0 = np.ascontiguousarray(np.broadcast_to(f_exact16, (codes.size, 19)))
    cfg = LevelConfig(dims=3, n=N, collision=MRT, nu=meta["nu"], bc_kind=tuple(meta["bc_kind"]))
    ref = np.ascontiguousarray(np.broadcast_to(f_exact16, (int(np.prod(N)), 19)))
    port.run(cfg, ref, ref.copy(), 1)
    post = ref[0]
    with zl.Context(_config(meta, storage, zl.ROUND_STOCHASTIC)) as ctx:
        ctx.set_level_nodes(0, codes)
        ctx.set_populations(0, codes, f0)
        assert np.array_equal(ctx.get_populations(0, None, codes.size), f0)  # the upload is exact
        ctx.set_block(0, *SHAPES[kernel])
        ctx.step_level(0)
        got = ctx.get_populations(0, None, codes.size)
    target = (post - w) * scale
    mean = (got.mean(0) - w) * scale
    moved = np.abs(target - _representable(target, storage)) > 1e-3 * _ulp(target, storage)
    assert moved.sum() >= 10  # most populations leave the 16-bit grid
    bias = np.abs(mean - target) / _ulp(target, storage)
    assert bias.max() <= 0.05, bias
