"""Faults injected on the host, none on the GPU: NaN-seeded populations are reported by the FP64
conservation check (ZL_ENAN) in every storage precision, calls on an out-of-range level or a
level without nodes are refused (ZL_EINVAL, ZL_ESTATE), and the context stays usable after each
refusal."""
import numpy as np
import pytest

from fixtures import load_lbm, solver_config

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", [0, 1, 2, 3])  # FP64, FP32, FP16, BF16
def test_nan_seeded_populations_are_reported(storage):
    import zllbm_b200 as zl
    meta, codes, f0, _ = load_lbm("tgv3d_mrt")
    with zl.Context(solver_config(meta, storage)) as ctx:
        ctx.set_level_nodes(0, codes)
        ctx.set_populations(0, codes, f0)
        assert np.all(np.isfinite(ctx.conservation(0)))
        bad = f0.copy()
        bad[len(bad) // 2, 3] = np.nan
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
