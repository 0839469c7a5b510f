"""Storage precision on the Taylor-Green vortex (zllbm_b200.tgv_accuracy), reduced size: FP32 /
FP16 / BF16 deviation storage against the FP64 run (the path bit-exact to the reference)."""
import pytest

pytestmark = pytest.mark.gpu


def test_tgv_storage_precision_small():
    from zllbm_b200.tgv_accuracy import run
    res = run(n=48, steps=400, checkpoints=2, log=lambda *a: None)
    st = res["storages"]
    assert max(st["f32"]["velocity_rel_l2_vs_f64"]) <= 1e-5
    assert max(st["f16"]["velocity_rel_l2_vs_f64"]) <= 5e-3
    assert max(st["bf16"]["velocity_rel_l2_vs_f64"]) <= 2e-2
    # the nonlinear transfer only adds dissipation: the FP64 run never keeps more energy than the
    # linear viscous decay
    kes, lin = res["kinetic_energy_f64"], res["kinetic_energy_linear_decay"]
    assert all(k <= l * 1.005 for k, l in zip(kes, lin))
