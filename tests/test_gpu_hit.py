"""The HIT closure pipeline on a small box: initial field, fine run, filtered training pairs,
tensor-core training, coarse Smagorinsky and learned runs.  The trained network must beat the
method without it (constant Smagorinsky, y = 1) on held-out pairs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_hit_initial_field_is_solenoidal_with_the_requested_rms():
    import torch
    from zllbm_b200.hit import energy_spectrum, hit_velocity
    n = 64
    u = hit_velocity(n, k0=4.0, u_rms=0.04, seed=7)
    g = u.reshape(n, n, n, 3).double()
    assert float(torch.sqrt((g * g).sum(-1).mean() / 3)) == pytest.approx(0.04, rel=1e-6)
    uh = torch.fft.fftn(g, dim=(0, 1, 2))
    k = torch.fft.fftfreq(n, 1.0 / n, device="cuda").double()
    div = k[None, None, :] * uh[..., 0] + k[None, :, None] * uh[..., 1] + k[:, None, None] * uh[..., 2]
    # FP32 rounding of the field leaves ~1e-7 relative noise in the spectral divergence
    assert float(div.abs().max()) < 1e-5 * float(uh.abs().max())
    e = energy_spectrum(u, n)
    assert 2 <= int(np.argmax(e)) <= 6
    assert e.sum() == pytest.approx(0.5 * 3 * 0.04 ** 2, rel=1e-6)


def test_hit_pipeline_small_box_network_beats_smagorinsky_a_priori():
    from zllbm_b200.hit import HitConfig, run
    cfg = HitConfig(fine=128, factor=4, nu_fine=0.002, coarse_steps=400, checkpoints=4, train_snapshots=2,
                    train_steps=300, batch=128 * 64, closure_every=4, calibrate_alpha=(0.8, 1.0),
                    calibrate_cs=(0.1,), test_realizations=2)
    res = run(cfg, log=lambda m: None)
    tr = res.training
    assert tr["val_loss"] < tr["val_loss_smagorinsky_y1"]
    assert tr["val_loss"] < tr["val_loss_best_constant"]
    for name in ("smagorinsky", "learned", "learned_calibrated", "learned_calibrated_every4"):
        assert res.errors[name]["error"] is not None
        assert np.isfinite(res.errors[name]["error"])
        assert res.mlups[name] > 0
        seeds = [r["seed"] for r in res.errors[name]["per_realization"]]
        assert seeds == [cfg.seed + 1000, cfg.seed + 2000]
        assert np.isfinite(res.errors[name]["error_std"])
    assert len(res.errors["learned_minus_smagorinsky_calibrated"]["per_realization"]) == 2
