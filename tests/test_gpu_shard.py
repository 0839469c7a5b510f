"""Slab sharding on the device (zl_set_level_halo, zl_halo_pack / zl_halo_unpack, zllbm_b200.shard):
a lattice split into 2 or 3 slabs of its last axis, one context per slab on one GPU, stepped by
the sharding schedule with the halo buffers routed between the contexts, equals the same lattice
in one context bit for bit (FP64 and FP32 storage; the step kernels' arithmetic does not depend on
where a node lies), for periodic and wall-bounded split axes, D3Q19 and D2Q9."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _config(dims, storage, periodic_split, coll):
    import zllbm_b200 as zl
    n = (24, 16, 20) if dims == 3 else (40, 36)
    kinds = [zl.BC_PERIODIC] * (2 * dims)
    vel = [(0.0, 0.0, 0.0)] * 6
    if not periodic_split:  # walls on the split axis, the high one moving
        kinds[2 * dims - 2] = kinds[2 * dims - 1] = zl.BC_BOUNCE_BACK
        vel[2 * dims - 1] = (0.05, 0.0, 0.0)
    lo = (1,) * dims
    hi = tuple(1 + n[a] for a in range(dims))
    cfg = zl.SolverConfig(lattice=zl.D3Q19 if dims == 3 else zl.D2Q9, collision=coll, storage=storage,
                          viscosity=0.02, rho0=1.0, bc_kind=tuple(kinds) + (0,) * (6 - 2 * dims),
                          bc_velocity=tuple(vel), domain_min=lo, domain_max=hi)
    return cfg


def _box(cfg):
    """(lo, n) of the context's level-0 box: unique nodes (periodic axes drop the duplicate plane)."""
    import zllbm_b200 as zl
    d = cfg.dims
    lo = tuple(cfg.domain_min[:d])
    n = tuple(cfg.domain_max[a] - cfg.domain_min[a] + (0 if cfg.bc_kind[2 * a] == zl.BC_PERIODIC else 1)
              for a in range(d))
    return lo, n


def _codes(dims, lo, n):
    import zllbm_b200 as zl
    return zl.box_codes(dims, lo, tuple(lo[a] + n[a] - 1 for a in range(dims)))


def _populations(cfg, codes, seed=5):
    """Seeded perturbation of the rest state per node, a function of the node's code only."""
    q = cfg.q
    w = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4) if q == 9 else np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
    rng = np.random.default_rng(seed)
    table = 1 + 0.05 * rng.standard_normal((int(codes.max()) + 1, q))
    return np.ascontiguousarray(w * table[codes.astype(np.int64)])


@pytest.mark.parametrize("storage", [0, 1])  # FP64, FP32
@pytest.mark.parametrize("periodic_split", [True, False])
@pytest.mark.parametrize("dims,world", [(3, 2), (3, 3), (2, 3)])
def test_slabs_equal_single_context(dims, world, periodic_split, storage):
    import zllbm_b200 as zl
    from zllbm_b200.shard import DeviceSlab, LocalRing, Ring, slab_range, split_planes
    cfg = _config(dims, storage, periodic_split, zl.MRT)
    glo, gn = _box(cfg)
    gcodes = _codes(dims, glo, gn)
    f0 = _populations(cfg, gcodes)
    steps = 8
    with zl.Context(cfg) as ctx:
        ctx.set_level_box(0, glo + (0,) * (3 - dims), gn + (1,) * (3 - dims))
        ctx.set_populations(0, gcodes, f0)
        ctx.advance(steps)
        ref = ctx.get_populations(0, gcodes)
    ref_by_code = dict(zip(gcodes.tolist(), range(gcodes.size)))

    planes = split_planes(cfg)
    slabs = []
    try:
        for r in range(world):
            lo, hi = slab_range(planes, r, world)
            slabs.append(DeviceSlab(cfg, lo, hi, Ring(r, world, periodic_split)))
        for s in slabs:
            codes = _codes(dims, s.box_lo, s.box_n)
            s.ctx.set_populations(0, codes, f0[[ref_by_code[c] for c in codes.tolist()]])
        ring = LocalRing(slabs, periodic_split, slabs[0].faces)
        for _ in range(steps // 2):
            ring.step_pair()
        for s in slabs:
            codes = _codes(dims, s.box_lo, s.box_n)
            got = s.ctx.get_populations(0, codes)
            want = ref[[ref_by_code[c] for c in codes.tolist()]]
            assert np.array_equal(got, want), (s.lo, s.hi, float(np.abs(got - want).max()))
    finally:
        for s in slabs:
            s.close()


def test_slab_mid_pair_read_back():
    """After an even step and its stage-0 swap, the populations read back (odd layout, boundary
    nodes reading the ghost planes) equal the single context's after one step."""
    import zllbm_b200 as zl
    from zllbm_b200.shard import DeviceSlab, LocalRing, Ring, slab_range, split_planes
    cfg = _config(3, 0, True, zl.MRT)
    glo, gn = _box(cfg)
    gcodes = _codes(3, glo, gn)
    f0 = _populations(cfg, gcodes)
    with zl.Context(cfg) as ctx:
        ctx.set_level_box(0, glo, gn)
        ctx.set_populations(0, gcodes, f0)
        ctx.step_level(0)
        ref = ctx.get_populations(0, gcodes)
    idx = dict(zip(gcodes.tolist(), range(gcodes.size)))
    slabs = [DeviceSlab(cfg, *slab_range(split_planes(cfg), r, 2), Ring(r, 2, True)) for r in range(2)]
    try:
        for s in slabs:
            codes = _codes(3, s.box_lo, s.box_n)
            s.ctx.set_populations(0, codes, f0[[idx[c] for c in codes.tolist()]])
        LocalRing(slabs, True, slabs[0].faces).step()
        for s in slabs:
            codes = _codes(3, s.box_lo, s.box_n)
            assert np.array_equal(s.ctx.get_populations(0, codes), ref[[idx[c] for c in codes.tolist()]])
    finally:
        for s in slabs:
            s.close()


def test_halo_errors():
    import zllbm_b200 as zl
    cfg = _config(3, 1, True, zl.MRT)
    lo, n = _box(cfg)
    with zl.Context(cfg) as ctx:
        ctx.set_level_box(0, lo, n)
        with pytest.raises(zl.ZlError):
            ctx.set_level_halo(0, 1 << 4)  # a periodic face
        with pytest.raises(zl.ZlError):
            ctx.halo_pack(0, 4, 0, 0)  # not a halo face
    cfg.bc_kind = cfg.bc_kind[:4] + (zl.BC_NONE, zl.BC_NONE)
    cfg.domain_max = cfg.domain_max[:2] + (cfg.domain_max[2] - 1,)
    lo, n = _box(cfg)
    with zl.Context(cfg) as ctx:
        ctx.set_level_box(0, lo, n)
        ctx.set_level_halo(0, 3 << 4)
        with pytest.raises(zl.ZlError):
            ctx.halo_pack(0, 4, 2, 0)  # bad stage
        with pytest.raises(zl.ZlError):
            ctx.set_level_halo(0, 1 << 6)  # no such face
        assert ctx.halo_bytes(0, 4) == 5 * n[0] * n[1] * 4


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("kernel,storage", [("pair", 1), ("pair", 2), ("row", 2), ("row", 3)])
def test_ring_slabs_take_full_box_kernels(kernel, storage, world):
    """Slabs of a periodic box (x and y periodic, both z faces connected) run the two-nodes-per-
    thread and one-warp-per-row kernels with z addressed through the ghost planes.  With round-to-
    nearest storage the row kernel equals the single context running it bit for bit.  The pair
    kernel hands the rows whose y or z neighbours wrap to the one-node update, which rounds
    differently in FP32: the single context does so for its z = 0 and z = n - 1 rows, the slabs
    (whose z neighbours never wrap) do not, so that case agrees to FP32 rounding only."""
    import zllbm_b200 as zl
    from zllbm_b200.shard import DeviceSlab, LocalRing, Ring, slab_range, split_planes
    n = (128, 8, 12)
    cfg = zl.SolverConfig(lattice=zl.D3Q19, collision=zl.MRT, storage=storage, viscosity=0.02, rho0=1.0,
                          bc_kind=(zl.BC_PERIODIC,) * 6, domain_min=(1, 1, 1), domain_max=tuple(1 + v for v in n),
                          storage_rounding=zl.ROUND_NEAREST)
    block = (-64, 1) if kernel == "pair" else (zl.BLOCK_ROW, 4)
    glo, gn = _box(cfg)
    gcodes = _codes(3, glo, gn)
    f0 = _populations(cfg, gcodes)
    steps = 6
    with zl.Context(cfg) as ctx:
        ctx.set_level_box(0, glo, gn)
        ctx.set_populations(0, gcodes, f0)
        ctx.set_block(0, *block)
        ctx.advance(steps)
        ref = ctx.get_populations(0, gcodes)
    idx = dict(zip(gcodes.tolist(), range(gcodes.size)))
    slabs = []
    try:
        for r in range(world):
            slabs.append(DeviceSlab(cfg, *slab_range(split_planes(cfg), r, world), Ring(r, world, True)))
        for s in slabs:
            codes = _codes(3, s.box_lo, s.box_n)
            s.ctx.set_populations(0, codes, f0[[idx[c] for c in codes.tolist()]])
            s.ctx.set_block(0, *block)  # refused unless the slab qualifies for the kernel
        ring = LocalRing(slabs, True, slabs[0].faces)
        for _ in range(steps // 2):
            ring.step_pair()
        for s in slabs:
            codes = _codes(3, s.box_lo, s.box_n)
            got, want = s.ctx.get_populations(0, codes), ref[[idx[c] for c in codes.tolist()]]
            if kernel == "row":
                assert np.array_equal(got, want), (s.lo, float(np.abs(got - want).max()))
            else:
                np.testing.assert_allclose(got, want, rtol=0, atol=2e-6)
    finally:
        for s in slabs:
            s.close()


def test_open_chain_slab_refuses_full_box_kernels():
    """An end slab of a wall-bounded axis has a missing-upstream face: only the general kernel runs it."""
    import zllbm_b200 as zl
    from zllbm_b200.shard import DeviceSlab, Ring, slab_range, split_planes
    cfg = _config(3, 1, False, zl.MRT)
    s = DeviceSlab(cfg, *slab_range(split_planes(cfg), 0, 2), Ring(0, 2, False))
    try:
        with pytest.raises(zl.ZlError):
            s.ctx.set_block(0, -64, 1)
    finally:
        s.close()


@pytest.mark.parametrize("world", [1, 2, 3])
@pytest.mark.parametrize("kernel,storage", [("scalar", 0), ("scalar", 1), ("pair", 1), ("row", 2)])
def test_overlapped_schedule_equals_plain(kernel, storage, world):
    """The overlapped schedule (interior planes stepped before the halo of the previous step is
    unpacked, zl_step_level_planes) equals the plain schedule bit for bit, on every step kernel."""
    import zllbm_b200 as zl
    from zllbm_b200.shard import DeviceSlab, LocalRing, Ring, slab_range, split_planes
    n = (128, 8, 21)
    cfg = zl.SolverConfig(lattice=zl.D3Q19, collision=zl.MRT, storage=storage, viscosity=0.02, rho0=1.0,
                          bc_kind=(zl.BC_PERIODIC,) * 6, domain_min=(1, 1, 1), domain_max=tuple(1 + v for v in n),
                          storage_rounding=zl.ROUND_NEAREST)
    block = {"scalar": None, "pair": (-64, 1), "row": (zl.BLOCK_ROW, 4)}[kernel]
    glo, gn = _box(cfg)
    gcodes = _codes(3, glo, gn)
    f0 = _populations(cfg, gcodes)
    idx = dict(zip(gcodes.tolist(), range(gcodes.size)))
    out = []
    for overlap in (False, True):
        slabs = []
        try:
            for r in range(world):
                slabs.append(DeviceSlab(cfg, *slab_range(split_planes(cfg), r, world), Ring(r, world, True)))
            for s in slabs:
                codes = _codes(3, s.box_lo, s.box_n)
                s.ctx.set_populations(0, codes, f0[[idx[c] for c in codes.tolist()]])
                if block:
                    s.ctx.set_block(0, *block)
            ring = LocalRing(slabs, True, slabs[0].faces, overlap=overlap)
            assert ring.overlap == overlap
            for _ in range(4):
                ring.step_pair()
            ring.flush()
            out.append([s.ctx.get_populations(0, _codes(3, s.box_lo, s.box_n)) for s in slabs])
        finally:
            for s in slabs:
                s.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_plane_steps_refused_where_they_do_not_apply():
    import zllbm_b200 as zl
    cfg = _config(2, 1, True, zl.MRT)
    lo, n = _box(cfg)
    with zl.Context(cfg) as ctx:
        ctx.set_level_box(0, lo + (0,), n + (1,))
        with pytest.raises(zl.ZlError):
            ctx.step_level_planes(0, 0, 1, True)  # D2Q9
    cfg = _config(3, 1, True, zl.MRT)
    lo, n = _box(cfg)
    with zl.Context(cfg) as ctx:
        ctx.set_level_box(0, lo, n)
        with pytest.raises(zl.ZlError):
            ctx.step_level_planes(0, n[2] - 1, 2, True)  # past the last plane
        ctx.step_level_planes(0, 0, n[2], True)  # a whole step in one call
