"""CUDA-graph replay of the sub-cycled step and the block-shape autotuner change no result.

A graph holds two background steps (every level back to the same population layout); odd step
counts finish with one direct step.  FP64 runs are compared bit for bit with the direct
(launch-by-launch) path and, where the step count matches, with the reference's own dumps.
Immersed-boundary runs are compared to 1e-12 (their node forces sum vertex shares in another order
than the reference).
"""
import numpy as np
import pytest

from test_gpu_amr import AMR, config, load_amr


def run(meta, z, storage, steps, graph=False, tune=False):
    import zllbm_b200 as zl
    levels = meta["levels"]
    with zl.Context(config(meta, storage)) as ctx:
        for lv in range(levels + 1):
            ctx.set_level_nodes(lv, z[f"codes{lv}"])
            ctx.set_populations(lv, z[f"codes{lv}"], z[f"f_before{lv}"])
        for lv in range(1, levels + 1):
            excluded = z[f"codes{lv - 1}"][(z[f"flags{lv - 1}"] & 4) != 0]
            ctx.set_level_interface(lv, z[f"c2f_fine{lv}"], z[f"f2c_coarse{lv - 1}"], excluded)
        if "ib" in meta:
            v = z["vertices_before"]
            ctx.ib_set_vertices(levels, v[:, 0:3], v[:, 3:6], v[:, 6])
        shapes = [ctx.autotune(lv, trials=2) for lv in range(levels + 1)] if tune else None
        ctx.set_graph(graph)
        # two calls: the second replays the graph captured by the first
        ctx.advance(steps // 2)
        ctx.advance(steps - steps // 2)
        pops = [ctx.get_populations(lv, z[f"codes{lv}"]) for lv in range(levels + 1)]
    return pops, shapes


def compare(a, b, ib):
    for x, y in zip(a, b):
        if ib:
            np.testing.assert_allclose(x, y, rtol=1e-12, atol=1e-15)
        else:
            assert np.array_equal(x, y)


@pytest.mark.gpu
@pytest.mark.parametrize("name", AMR)
def test_graph_replay_matches_direct_fp64(name):
    import zllbm_b200 as zl
    meta, z = load_amr(name)
    ib = "ib" in meta
    for steps in (meta["steps"], 5):
        direct, _ = run(meta, z, zl.STORAGE_F64, steps)
        graphed, _ = run(meta, z, zl.STORAGE_F64, steps, graph=True)
        compare(graphed, direct, ib)
        if steps == meta["steps"]:
            compare(graphed, [z[f"f_after{lv}"] for lv in range(meta["levels"] + 1)], ib)


@pytest.mark.gpu
@pytest.mark.parametrize("name", AMR)
def test_graph_replay_matches_direct_fp32(name):
    import zllbm_b200 as zl
    meta, z = load_amr(name)
    direct, _ = run(meta, z, zl.STORAGE_F32, 6)
    graphed, _ = run(meta, z, zl.STORAGE_F32, 6, graph=True)
    compare(graphed, direct, "ib" in meta)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["amr2d_l2", "amr3d_l1"])
def test_autotuned_block_shape_keeps_results(name):
    import zllbm_b200 as zl
    meta, z = load_amr(name)
    direct, _ = run(meta, z, zl.STORAGE_F64, meta["steps"])
    tuned, shapes = run(meta, z, zl.STORAGE_F64, meta["steps"], graph=True, tune=True)
    compare(tuned, direct, False)
    for bx, by in shapes:
        assert bx >= 32 and by >= 1 and bx * by <= 256


@pytest.mark.gpu
def test_autotune_on_periodic_box_keeps_results():
    """A 3D periodic TGV box (odd extents, so blocks overhang on x and y) tuned then stepped."""
    import zllbm_b200 as zl
    from fixtures import load_lbm, solver_config
    meta, codes, f0, f1 = load_lbm("tgv3d_mrt")
    results = []
    for tune in (False, True):
        with zl.Context(solver_config(meta, zl.STORAGE_F64)) as ctx:
            ctx.set_level_nodes(0, codes)
            ctx.set_populations(0, codes, f0)
            if tune:
                ctx.autotune(0, trials=2)
            ctx.set_graph(True)
            ctx.advance(meta["steps"])
            results.append(ctx.get_populations(0, codes))
    assert np.array_equal(results[0], results[1])
    assert np.array_equal(results[1], f1)


@pytest.mark.gpu
def test_graph_recaptured_after_direct_step():
    """A direct zl_step_level between zl_advance calls flips the layout; the replayed graph must
    follow it (and a new node set must drop the old graph)."""
    import zllbm_b200 as zl
    from fixtures import load_lbm, solver_config
    meta, codes, f0, _ = load_lbm("cavity2d_mrt")
    results = []
    for graph in (False, True):
        with zl.Context(solver_config(meta, zl.STORAGE_F64)) as ctx:
            ctx.set_level_nodes(0, codes)
            ctx.set_populations(0, codes, f0)
            ctx.set_graph(graph)
            ctx.advance(4)
            ctx.step_level(0)
            ctx.advance(4)
            ctx.advance(3)
            ctx.set_level_nodes(0, codes)
            ctx.set_populations(0, codes, f0)
            ctx.advance(6)
            results.append(ctx.get_populations(0, codes))
    assert np.array_equal(results[0], results[1])


@pytest.mark.gpu
@pytest.mark.parametrize("name", AMR)
def test_batched_levels_match_one_launch_per_level(name):
    """The sub-cycled order on one stream with one launch per level step, with consecutive
    independent level steps sharing one launch (batching), and on per-level streams ordered by the
    levels each operation touches (default), directly and replayed from a graph: FP64 results
    agree bit for bit."""
    import zllbm_b200 as zl
    meta, z = load_amr(name)
    levels = meta["levels"]
    out = []
    modes = [(False, False, False), (False, True, False), (True, False, False), (True, False, True)]
    for streams, batched, graph in modes:
        with zl.Context(config(meta, zl.STORAGE_F64)) as ctx:
            for lv in range(levels + 1):
                ctx.set_level_nodes(lv, z[f"codes{lv}"])
                ctx.set_populations(lv, z[f"codes{lv}"], z[f"f_before{lv}"])
            for lv in range(1, levels + 1):
                excluded = z[f"codes{lv - 1}"][(z[f"flags{lv - 1}"] & 4) != 0]
                ctx.set_level_interface(lv, z[f"c2f_fine{lv}"], z[f"f2c_coarse{lv - 1}"], excluded)
            if "ib" in meta:
                v = z["vertices_before"]
                ctx.ib_set_vertices(levels, v[:, 0:3], v[:, 3:6], v[:, 6])
            ctx.set_level_streams(streams)
            ctx.set_batching(batched)
            ctx.set_graph(graph)
            ctx.advance(meta["steps"] + 1)
            out.append([ctx.get_populations(lv, z[f"codes{lv}"]) for lv in range(levels + 1)])
    for o in out[1:]:
        compare(o, out[0], "ib" in meta)


def _amr_ctx(meta, z, storage):
    import zllbm_b200 as zl
    levels = meta["levels"]
    ctx = zl.Context(config(meta, storage))
    for lv in range(levels + 1):
        ctx.set_level_nodes(lv, z[f"codes{lv}"])
        ctx.set_populations(lv, z[f"codes{lv}"], z[f"f_before{lv}"])
    for lv in range(1, levels + 1):
        excluded = z[f"codes{lv - 1}"][(z[f"flags{lv - 1}"] & 4) != 0]
        ctx.set_level_interface(lv, z[f"c2f_fine{lv}"], z[f"f2c_coarse{lv - 1}"], excluded)
    return ctx


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["amr2d_l1", "amr3d_l1"])
def test_interface_interpolation_is_the_mean_of_two_transfers(name):
    """zl_interpolate_interface writes 0.5 (last transfer + transfer from the coarse state now)
    into the explosion targets (FP64, bit for bit)."""
    import zllbm_b200 as zl
    meta, z = load_amr(name)
    ghosts = z["c2f_fine1"]
    seq = lambda ctx: (ctx.step_level(0), ctx.step_level(1), ctx.step_level(1), ctx.transfer_levels(1),
                       ctx.step_level(0), ctx.step_level(1))
    with _amr_ctx(meta, z, zl.STORAGE_F64) as a, _amr_ctx(meta, z, zl.STORAGE_F64) as b:
        a.step_level(0), a.step_level(1), a.step_level(1), a.transfer_levels(1)
        b.step_level(0), b.step_level(1), b.step_level(1), b.transfer_levels(1)
        last = a.get_populations(1, ghosts)
        for ctx in (a, b):
            ctx.step_level(0)
            ctx.step_level(1)
        a.interpolate_interface(1)
        b.transfer_levels(1)
        mean = a.get_populations(1, ghosts)
        now = b.get_populations(1, ghosts)
    assert np.array_equal(mean, 0.5 * (last + now))
    assert not np.array_equal(mean, now)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["amr2d_l1", "amr3d_l1"])
def test_temporal_interpolation_in_advance_follows_the_public_steps(name):
    """zl_advance with time interpolation equals, bit for bit, the public calls it stands for:
    coarse step, fine step, interface interpolation, fine step, transfer; and it changes the run."""
    import zllbm_b200 as zl
    meta, z = load_amr(name)
    codes = [z["codes0"], z["codes1"]]
    res = {}
    for mode in ("advance", "manual", "plain"):
        with _amr_ctx(meta, z, zl.STORAGE_F64) as ctx:
            ctx.advance(1)  # ends with a transfer
            if mode == "advance":
                ctx.set_temporal_interpolation(True)
                ctx.advance(2)
            elif mode == "manual":
                for _ in range(2):
                    ctx.step_level(0)
                    ctx.step_level(1)
                    ctx.interpolate_interface(1)
                    ctx.step_level(1)
                    ctx.transfer_levels(1)
            else:
                ctx.advance(2)
            res[mode] = [ctx.get_populations(lv, codes[lv]) for lv in (0, 1)]
    for a, b in zip(res["advance"], res["manual"]):
        assert np.array_equal(a, b)
    assert not np.array_equal(res["advance"][1], res["plain"][1])

@pytest.mark.gpu
@pytest.mark.parametrize("storage,tol", [(1, 1e-5), (2, 5e-3), (3, 5e-2)])
@pytest.mark.parametrize("coll", ["tgv3d_mrt", "tgv3d_srt"])
def test_two_nodes_per_thread_kernel(coll, storage, tol):
    """The packed-pair kernel against the reference dump (same tolerances as the scalar kernel)
    and against the scalar kernel (FP32: 1e-6)."""
    import zllbm_b200 as zl
    from fixtures import load_lbm, solver_config
    meta, codes, f0, f1 = load_lbm(coll)
    out = []
    for shape in ((128, 1), (-64, 1), (-32, 2)):
        with zl.Context(solver_config(meta, storage)) as ctx:
            ctx.set_level_nodes(0, codes)
            ctx.set_populations(0, codes, f0)
            ctx.set_block(0, *shape)
            ctx.advance(meta["steps"])
            out.append(ctx.get_populations(0, codes))
    w = np.abs(f1).max()
    for got in out[1:]:
        if storage == 1:
            assert np.abs(got - f1).max() <= tol * w
            assert np.abs(got - out[0]).max() <= 1e-6 * w
        else:
            from test_gpu_parity import velocity
            ue, ug = velocity(meta, f1), velocity(meta, got)
            assert np.linalg.norm(ug - ue) / np.linalg.norm(ue) <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("storage,tol", [(1, 1e-5), (2, 5e-3), (3, 5e-2)])
@pytest.mark.parametrize("coll", ["mrt", "srt"])
def test_two_nodes_per_thread_kernel_even_rows(coll, storage, tol, port):
    """Rows of even length take the packed-pair accesses (the fixtures above have odd rows and
    fall back to the scalar kernel): against the oracle restatement over 24 x 16 x 12 periodic
    nodes (same tolerances as the scalar kernel) and against the scalar kernel (FP32: 1e-6)."""
    import zllbm_b200 as zl
    from fixtures import grid_order, solver_config
    from oracle.port import BC_PERIODIC, MRT, SRT, LevelConfig, tgv_init
    from test_gpu_parity import velocity
    cfg = LevelConfig(dims=3, n=(25, 17, 13), collision=MRT if coll == "mrt" else SRT, nu=0.05 / 3,
                      bc_kind=(BC_PERIODIC,) * 6)
    steps = 21
    f = np.ascontiguousarray(tgv_init(cfg, 0.05, port).reshape(-1, cfg.q))
    codes = zl.box_codes(3, [1, 1, 1], list(cfg.n))
    lin = grid_order(codes, 3, cfg.n)
    f0 = f[lin].copy()
    port.run(cfg, f, f.copy(), steps)
    f1 = f[lin]
    meta = dict(dims=3, n=list(cfg.n), collision=cfg.collision, nu=cfg.nu, rho0=cfg.rho0,
                bc_kind=list(cfg.bc_kind), bc_vel=[list(v) for v in cfg.bc_vel], steps=steps)
    out = []
    for shape in ((128, 1), (-64, 1), (-32, 2), (-128, 1)):
        with zl.Context(solver_config(meta, storage)) as ctx:
            ctx.set_level_nodes(0, codes)
            ctx.set_populations(0, codes, f0)
            ctx.set_block(0, *shape)
            ctx.advance(steps)
            out.append(ctx.get_populations(0, codes))
    w = np.abs(f1).max()
    for got in out[1:]:
        if storage == 1:
            assert np.abs(got - f1).max() <= tol * w
            assert np.abs(got - out[0]).max() <= 1e-6 * w
        else:
            ue, ug = velocity(meta, f1), velocity(meta, got)
            assert np.linalg.norm(ug - ue) / np.linalg.norm(ue) <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("storage,tol", [(2, 5e-3), (3, 5e-2)])
@pytest.mark.parametrize("coll", ["mrt", "srt"])
@pytest.mark.parametrize("n", [(129, 9, 8), (257, 8, 8)])
def test_row_kernel(n, coll, storage, tol, port):
    """The one-warp-per-row kernel (128- and 256-node periodic rows, 1, 2 and 4 rows per block,
    the last block partly empty) against the oracle restatement after 13 steps (same tolerances
    as the scalar kernel) and against the two-nodes-per-thread kernel after two steps, bit for
    bit on the nodes whose populations depend only on rows the pair kernel updates with the same
    packed collision (its wrapped edge rows take the scalar kernel, which rounds differently)."""
    import zllbm_b200 as zl
    from fixtures import grid_order, solver_config
    from oracle.port import BC_PERIODIC, MRT, SRT, LevelConfig, morton_decode, tgv_init
    from test_gpu_parity import velocity
    cfg = LevelConfig(dims=3, n=n, collision=MRT if coll == "mrt" else SRT, nu=0.05 / 3,
                      bc_kind=(BC_PERIODIC,) * 6)
    steps = 13
    f = np.ascontiguousarray(tgv_init(cfg, 0.05, port).reshape(-1, cfg.q))
    codes = zl.box_codes(3, [1, 1, 1], list(cfg.n))
    lin = grid_order(codes, 3, cfg.n)
    f0 = f[lin].copy()
    port.run(cfg, f, f.copy(), steps)
    f1 = f[lin]
    meta = dict(dims=3, n=list(cfg.n), collision=cfg.collision, nu=cfg.nu, rho0=cfg.rho0,
                bc_kind=list(cfg.bc_kind), bc_vel=[list(v) for v in cfg.bc_vel], steps=steps)

    def run(shape, k):
        cfg = solver_config(meta, storage)
        cfg.storage_rounding = zl.ROUND_NEAREST  # both kernels round the same way (bit-for-bit check)
        with zl.Context(cfg) as ctx:
            ctx.set_level_nodes(0, codes)
            ctx.set_populations(0, codes, f0)
            ctx.set_block(0, *shape)
            ctx.advance(k)
            return ctx.get_populations(0, codes)

    rows = [(zl.BLOCK_ROW, 4), (zl.BLOCK_ROW, 2), (zl.BLOCK_ROW, 1)]
    ue = velocity(meta, f1)
    out = [run(shape, steps) for shape in rows]
    for got in out:
        ug = velocity(meta, got)
        assert np.linalg.norm(ug - ue) / np.linalg.norm(ue) <= tol
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])
    # two steps (even, odd): node x's populations come from the odd-step collisions of its
    # neighbours, whose inputs the neighbours' neighbours wrote in the even step
    idx = morton_decode(codes, 3) - 1
    uniq = [v - 1 for v in n]
    inner = np.ones(len(codes), dtype=bool)
    for a in (1, 2):
        inner &= (idx[:, a] >= 3) & (idx[:, a] <= uniq[a] - 4)
    assert inner.sum() >= uniq[0]
    pair2 = run((-64, 1), 2)
    row2 = run(rows[0], 2)
    assert np.array_equal(row2[inner], pair2[inner])


@pytest.mark.gpu
def test_row_kernel_refused_where_it_does_not_apply():
    import zllbm_b200 as zl
    from fixtures import load_lbm, solver_config
    meta, codes, f0, _ = load_lbm("tgv3d_mrt")  # 10-node rows
    for storage in (1, 2):
        with zl.Context(solver_config(meta, storage)) as ctx:
            ctx.set_level_nodes(0, codes)
            with pytest.raises(zl.ZlError):
                ctx.set_block(0, zl.BLOCK_ROW, 4)
