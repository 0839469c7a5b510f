"""Analytic checks of the restated step (the oracle, pinned bit for bit to the reference): a uniform
equilibrium stays unchanged, and a body-force-driven channel between bounce-back walls reaches
the Poiseuille profile (constant curvature -g / nu, symmetric, uniform along the flow)."""
import numpy as np
import pytest

from oracle.port import BC_BOUNCE_BACK, BC_PERIODIC, MRT, SRT, LevelConfig


@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("coll", [SRT, MRT])
def test_uniform_equilibrium_is_invariant(dims, coll, port):
    n = (9, 7, 5)[:dims]
    cfg = LevelConfig(dims=dims, n=n, collision=coll, nu=0.03, bc_kind=(BC_PERIODIC,) * (2 * dims) + (0,) * (6 - 2 * dims))
    u = (0.05, -0.02, 0.01)[:dims]
    feq = port.feq(dims, 1.02, u)
    f = np.tile(feq, (int(np.prod(n)), 1))
    port.run(cfg, f, f.copy(), 20)
    np.testing.assert_allclose(f, np.broadcast_to(feq, f.shape), rtol=0, atol=1e-15)
    rho, vel = port.macros(cfg, f)
    np.testing.assert_allclose(rho, 1.02, rtol=1e-14)
    np.testing.assert_allclose(vel, np.broadcast_to(u, vel.shape), atol=1e-15)


@pytest.mark.parametrize("coll", [SRT, MRT])
def test_body_force_channel_reaches_poiseuille(coll, port):
    nu, g, ny = 0.1, 1e-6, 17  # stored nodes across the channel; walls on the first and last row
    cfg = LevelConfig(dims=2, n=(4, ny), collision=coll, nu=nu, force=(g, 0.0),
                      bc_kind=(BC_PERIODIC, BC_PERIODIC, BC_BOUNCE_BACK, BC_BOUNCE_BACK, 0, 0))
    f = np.tile(port.feq(2, 1.0, (0.0, 0.0)), (4 * ny, 1))
    fc = f.copy()
    port.run(cfg, f, fc, 6000)
    _, u_prev = port.macros(cfg, f)
    port.run(cfg, f, fc, 500)
    _, u = port.macros(cfg, f)
    ux = u[:, 0].reshape(ny, 4)
    assert np.abs(u - u_prev).max() < 1e-6 * ux.max()  # steady
    assert np.abs(u[:, 1]).max() < 1e-6 * ux.max()  # no cross flow
    np.testing.assert_allclose(ux, ux[:, :1].repeat(4, 1), rtol=1e-12, atol=1e-18)  # uniform along x
    prof = ux[:, 0]
    np.testing.assert_allclose(prof, prof[::-1], rtol=1e-9)  # symmetric about the centre line
    # constant curvature u'' = -g / nu, centred on rows 2 .. ny - 3 (wall rows and their
    # neighbours excluded)
    curv = prof[3:-1] - 2.0 * prof[2:-2] + prof[1:-3]
    np.testing.assert_allclose(curv, -g / nu, rtol=2e-3)


def _tgv_viscosity_ratio(port, dims, coll, cells, steps, nu=0.02, u0=0.005):
    """Effective over nominal viscosity from the kinetic-energy decay of a nearly linear TGV,
    E(t) = E(0) exp(-2 nu |k|^2 t) with |k|^2 = dims (2 pi / cells)^2."""
    import math

    from oracle.port import tgv_init
    n = (cells + 1,) * dims
    cfg = LevelConfig(dims=dims, n=n, collision=coll, nu=nu, bc_kind=(BC_PERIODIC,) * (2 * dims) + (0,) * (6 - 2 * dims))
    f = tgv_init(cfg, u0, port).reshape(-1, cfg.q)

    def energy():
        _, u = port.macros(cfg, f)
        g = u.reshape(tuple(reversed(n)) + (dims,))[(slice(0, cells),) * dims]  # unique nodes
        return 0.5 * (g ** 2).sum(-1).mean()

    e0 = energy()
    port.run(cfg, f, f.copy(), steps)
    k2 = dims * (2 * math.pi / cells) ** 2
    return -math.log(energy() / e0) / (2 * steps * k2) / nu


@pytest.mark.parametrize("dims,coll,cells,steps", [(2, SRT, 24, 200), (2, MRT, 24, 200), (3, SRT, 16, 100)])
def test_tgv_decay_converges_at_second_order(dims, coll, cells, steps, port):
    coarse = _tgv_viscosity_ratio(port, dims, coll, cells, steps) - 1.0
    fine = _tgv_viscosity_ratio(port, dims, coll, 2 * cells, 4 * steps) - 1.0  # same physical time
    assert abs(fine) < 0.025
    assert 3.0 < coarse / fine < 5.0  # error / 4 per halving of the spacing
