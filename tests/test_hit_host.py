"""Host side of the closure metric ("learned vs Smagorinsky LES error"): the shell spectrum and the
log-spectrum error, on CPU tensors with known answers."""
import math

import numpy as np
import pytest


def test_energy_spectrum_of_one_mode_and_parseval():
    import torch
    from zllbm_b200.hit import energy_spectrum
    n, kx, amp = 16, 3, 0.02
    x = 2 * math.pi * torch.arange(n, dtype=torch.float64) / n
    z, y, xx = torch.meshgrid(x, x, x, indexing="ij")
    u = torch.zeros(n, n, n, 3, dtype=torch.float64)
    u[..., 1] = amp * torch.sin(kx * xx)  # shear wave u_y(x), solenoidal
    e = energy_spectrum(u.reshape(-1, 3), n)
    assert e.shape == (n // 2 + 1,)
    assert int(np.argmax(e)) == kx
    assert e[kx] == pytest.approx(0.5 * amp * amp / 2, rel=1e-12)  # 0.5 <u^2>, <sin^2> = 1/2
    assert e.sum() - e[kx] == pytest.approx(0.0, abs=1e-20)


def test_spectrum_error_is_rms_log_ratio():
    from zllbm_b200.hit import spectrum_error
    ref = np.array([0.0, 1.0, 0.5, 0.25, 0.125])
    assert spectrum_error(ref, ref, 4) == 0.0
    assert spectrum_error(ref * math.e, ref, 4) == pytest.approx(1.0, rel=1e-12)
    # shell 0 and shells above k_max are ignored
    other = ref.copy()
    other[0], other[4] = 7.0, 9.0
    assert spectrum_error(other, ref, 3) == 0.0
