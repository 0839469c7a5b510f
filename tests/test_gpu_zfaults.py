"""Faults injected on the host, none on the GPU: NaN-seeded populations are reported by the FP64
conservation check (ZL_ENAN) in every storage precision, calls on an out-of-range level or a
level without nodes are refused (ZL_EINVAL, ZL_ESTATE), and the context stays usable after each
refusal."""
import numpy as np
import pytest

from fixtures import load_lbm, solver_config

pytestmark = pytest.mark.gpu


def _duplicate_plane_rows(meta, codes):
    """Rows of the node list that lie on the duplicated maximum plane of a periodic axis."""
    import zllbm_b200 as zl
    from oracle.port import morton_decode
    dims = meta["dims"]
    idx = morton_decode(codes, dims) - 1
    dup = np.zeros(len(codes), dtype=bool)
    for a in range(dims):
        if meta["bc_kind"][2 * a] == zl.BC_PERIODIC:
            dup |= idx[:, a] == meta["n"][a] - 1
    return dup


@pytest.mark.parametrize("storage", [0, 1, 2, 3])  # FP64, FP32, FP16, BF16
def test_nan_seeded_populations_are_reported(storage):
    import zllbm_b200 as zl
    meta, codes, f0, _ = load_lbm("tgv3d_mrt")
    with zl.Context(solver_config(meta, storage)) as ctx:
        ctx.set_level_nodes(0, codes)
        ctx.set_populations(0, codes, f0)
        assert np.all(np.isfinite(ctx.conservation(0)))
        bad = f0.copy()
        interior = np.flatnonzero(~_duplicate_plane_rows(meta, codes))
        bad[interior[len(interior) // 2], 3] = np.nan
        ctx.set_populations(0, codes, bad)
        with pytest.raises(zl.ZlError) as e:
            ctx.conservation(0)
        assert e.value.code == -5
        ctx.step_level(0)  # the step runs; the non-finite value spreads and stays reported
        with pytest.raises(zl.ZlError) as e:
            ctx.conservation(0)
        assert e.value.code == -5
        ctx.set_populations(0, codes, f0)
        assert np.all(np.isfinite(ctx.conservation(0)))


def test_bad_levels_are_refused_and_the_context_stays_usable():
    import zllbm_b200 as zl
    meta, codes, f0, _ = load_lbm("tgv3d_mrt")
    with zl.Context(solver_config(meta, zl.STORAGE_F64)) as ctx:
        with pytest.raises(zl.ZlError) as e:
            ctx.step_level(3)  # max_level is 0
        assert e.value.code == -1
        with pytest.raises(zl.ZlError) as e:
            ctx.conservation(0)  # no nodes yet
        assert e.value.code == -6
        ctx.set_level_nodes(0, codes)
        ctx.set_populations(0, codes, f0)
        ctx.advance(2)
        assert np.all(np.isfinite(ctx.conservation(0)))


@pytest.mark.parametrize("storage", [0, 1, 2, 3])  # FP64, FP32, FP16, BF16
def test_disagreeing_duplicate_planes_take_the_minimum_plane(storage):
    """The reference stores a periodic axis's maximum plane as a copy of its minimum plane
    (grid/grid_manager3d.cpp:106-112); the device stores that node once.  When the caller's two
    copies disagree, the minimum-plane copy is the one kept, in every storage precision."""
    import zllbm_b200 as zl
    meta, codes, f0, _ = load_lbm("tgv3d_mrt")
    dup = _duplicate_plane_rows(meta, codes)
    assert dup.any() and not dup.all()
    with zl.Context(solver_config(meta, storage)) as ctx:
        ctx.set_level_nodes(0, codes)
        ctx.set_populations(0, codes, f0)
        want = ctx.get_populations(0, codes)
        for perturb in (np.nan, 0.5):
            bad = f0.copy()
            bad[dup] = perturb if np.isnan(perturb) else f0[dup] * perturb
            ctx.set_populations(0, codes, bad)
            got = ctx.get_populations(0, codes)
            assert np.array_equal(got, want), perturb
            assert np.all(np.isfinite(ctx.conservation(0)))
