"""CPU checks of the learned-closure oracle: BF16 rounding, GELU, backward formulas (finite
differences), the Smagorinsky feature against the C restatement of the reference's model, and the
box filter / training-pair construction on small analytic fields."""
import numpy as np
import pytest

from oracle import closure as C


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    x = np.random.default_rng(0).normal(size=4096).astype(np.float32) * np.float32(3.0)
    x[:4] = [0.0, -0.0, 1e-30, 65504.0]
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(C.bf16(x), ref)


def test_gelu_is_the_tanh_form():
    torch = pytest.importorskip("torch")
    z = np.linspace(-8, 8, 257)
    ref = torch.nn.functional.gelu(torch.from_numpy(z), approximate="tanh").numpy()
    np.testing.assert_allclose(C.gelu(z), ref, rtol=1e-13, atol=1e-15)
    h = 1e-6
    np.testing.assert_allclose(C.gelu_grad(z), (C.gelu(z + h) - C.gelu(z - h)) / (2 * h), rtol=1e-6, atol=1e-8)


def test_backward_matches_finite_differences():
    net = C.Mlp.random(1)
    x = np.random.default_rng(2).normal(size=(64, 24))
    t = np.random.default_rng(3).uniform(0, 2, 64)
    _, g = net.gradients(x, t, rounding=False)
    rng = np.random.default_rng(4)
    for name in ("w1", "b1", "w2", "b2", "w3", "b3"):
        base = np.array(getattr(net, name), dtype=np.float64)
        for _ in range(4):
            idx = tuple(rng.integers(0, s) for s in base.shape)
            h = 1e-4
            vals = []
            for sgn in (1, -1):
                v = base.copy()
                v[idx] += sgn * h
                setattr(net, name, v)
                y, _ = net.forward(x, rounding=False)
                vals.append(((y - t) ** 2).mean())
            setattr(net, name, base)
            fd = (vals[0] - vals[1]) / (2 * h)
            an = np.asarray(g[name])[idx]
            assert abs(fd - an) <= 1e-6 + 1e-5 * abs(an), (name, idx, fd, an)


def test_smagorinsky_feature_matches_reference_model(port):
    """Feature 24 is the reference's Smagorinsky increment (lbm_les_smagorinsky.cpp:22-94) at
    Cs = 0.1, evaluated here and by the C restatement of the reference."""
    rng = np.random.default_rng(5)
    rho = 1.0 + 0.01 * rng.normal(size=8)
    u = 0.05 * rng.normal(size=(8, 3))
    feq = C.feq19(rho, u)
    f = feq * (1.0 + 1e-3 * rng.normal(size=feq.shape))
    tau0 = 0.52
    x = C.node_features(f, tau0)
    for i in range(8):
        ref = port.smag_tau_sgs(3, f[i], port.feq(3, float(f[i].sum()), (f[i] @ C.C19) / f[i].sum()), tau0, 1.0, 0.1)
        assert x[i, 23] == pytest.approx(ref, rel=1e-10, abs=1e-15)


def test_features_of_equilibrium_are_zero():
    rho = np.array([1.0, 1.02])
    u = np.array([[0.01, -0.02, 0.03], [0.0, 0.0, 0.0]])
    x = C.node_features(C.feq19(rho, u), 0.6)
    np.testing.assert_allclose(x, 0.0, atol=1e-15)


def test_filter_of_uniform_flow_and_zero_target():
    """A uniform equilibrium flow filters to itself and has no subgrid stress (target 0)."""
    n = (8, 8, 8)
    rho = np.full(512, 1.01)
    u = np.tile([0.02, -0.01, 0.005], (512, 1))
    filt = C.box_filter(C.feq19(rho, u), n, 2)
    np.testing.assert_allclose(filt[:, 0], 1.01)
    np.testing.assert_allclose(filt[:, 1:4], np.tile([0.02, -0.01, 0.005], (64, 1)), atol=1e-15)
    np.testing.assert_allclose(filt[:, 10:], 0.0, atol=1e-15)
    x, y = C.training_pairs(filt, (4, 4, 4), 0.52, 0.505, 2)
    assert np.all(y == 0.0)


def test_subgrid_stress_of_a_resolved_shear_is_zero():
    """For u_x = a y, u_y = b x the box-filtered cross stress <u_x u_y> - <u_x><u_y> = a b cov(x, y)
    vanishes: x and y are independent over a box."""
    nx = 16
    yy = np.repeat(np.arange(nx), nx)  # y index of each node of a 16 x 16 x 1 plane (x fastest)
    xx = np.tile(np.arange(nx), nx)
    u = np.zeros((nx * nx, 3))
    u[:, 0] = 1e-3 * yy
    u[:, 1] = 2e-3 * xx
    uu = np.stack([u[:, a] * u[:, b] for a, b in C.PAIRS], axis=1)
    g = np.concatenate([u, uu], axis=1).reshape(1, nx // 4, 4, nx // 4, 4, 9).mean(axis=(2, 4)).reshape(-1, 9)
    tau_xy = g[:, 3 + 3] - g[:, 0] * g[:, 1]
    np.testing.assert_allclose(tau_xy, 0.0, atol=1e-18)


def test_adam_first_step_moves_by_lr_times_sign():
    net = C.Mlp.random(7)
    opt = C.Adam(net)
    before = net.w2.copy()
    g = {k: np.ones_like(np.asarray(getattr(net, k), dtype=np.float64)) * 0.3 for k in opt.m}
    opt.step(g, 1e-2)
    np.testing.assert_allclose(net.w2, before - 1e-2, rtol=0, atol=1e-6)


def test_bf16_gelu_constants_and_accuracy():
    assert C.bf16(np.float32(C.GELU_A)) == np.float32(C.A_BF16)
    assert C.bf16(np.float32(C.GELU_K)) == np.float32(C.K_BF16)
    z = np.linspace(-6, 6, 1001)
    err = np.abs(C.gelu_bf16(z) - C.gelu(z))
    assert err.max() < 0.03 * max(1.0, np.abs(z).max()) and np.median(err) < 5e-3


def test_delta_kernels_moment_conditions():
    """Both immersed-boundary kernels are partitions of unity with zero first moment; the
    three-point kernel also has sum phi^2 = 1/2 (Roma, Peskin and Berger 1999)."""
    from oracle import ib
    for x in np.linspace(0.0, 1.0, 41):
        for width in (3, 4):
            nodes, w = ib.stencil(10.0 + x, width)
            assert w.sum() == pytest.approx(1.0, abs=1e-14)
            assert ((10.0 + x - nodes) * w).sum() == pytest.approx(0.0, abs=1e-14)
        nodes, w = ib.stencil(10.0 + x, 3)
        assert (w ** 2).sum() == pytest.approx(0.5, abs=1e-14)
    assert ib.delta_three(np.array([1.5, 2.0]))[0] == pytest.approx(0.0, abs=1e-15)
