"""ORACLE — test infrastructure only.

CPU restatement of the learned LES closure: the node features, the MLP 24 -> 64 -> 64 -> 1
(tanh-form GELU) forward and backward passes with the device's BF16 rounding points, the Adam
update, the box filter of fine-level populations and the training pairs built from it.  The
tests compare the device kernels (tensor-core forward/backward, fused in-collision inference,
filter and pair kernels) against these functions.  Nothing in the product imports this module.

The closure has no counterpart in the reference (it hard-wires Smagorinsky,
lbm_project/les_models/lbm_les_smagorinsky.cpp:22-94); its relaxation-time formula is the
reference's Smagorinsky increment with the constant C = 18 c taken per node from the network:

    tau_eff = tau0 + 0.5 * (sqrt(tau0^2 + 18 c sqrt(2 Pi:Pi)) - tau0),  c = 0.01 * clamp(y, 0, 8)

so y = 1 reproduces Smagorinsky with Cs = 0.1.

Rounding points shared with the device (everything else FP32):
  * network inputs x_hat = (x - mean) * inv_std, W1, A1 = gelu(Z1), W2 are BF16 tensor-core operands,
    and so are the biases b1, b2 (they ride on a ones column of the products);
  * inference evaluates GELU on packed BF16 pairs, every operation rounded to BF16 (gelu_bf16);
    training uses the FP32 GELU;
  * backward: dZ2 and dZ1 are BF16 operands of the gradient products (the bias gradients come
    from a ones column of those products, so they sum the BF16 values); dZ1 uses the FP32 dA1.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID = 24, 64
GELU_K = 0.7978845608028654  # sqrt(2 / pi)
GELU_A = 0.044715
C_UNIT = 0.01                # c = C_UNIT * y  (y = 1 <=> Smagorinsky Cs = 0.1)
Y_MAX = 8.0
DEN_MIN = 1e-30  # <M:M> below this (|S| ~ 1e-8) fits no constant

# D3Q19 velocities and MRT moment basis in the reference's order (lbm_d3q19.h:18-46, :98-167)
C19 = np.array([(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (1, 1, 0),
                (-1, 1, 0), (1, -1, 0), (-1, -1, 0), (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1), (0, 1, 1),
                (0, -1, 1), (0, 1, -1), (0, -1, -1)], dtype=np.float64)
W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
M19 = np.array([
    [1] * 19,
    [-30, -11, -11, -11, -11, -11, -11, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8],
    [12, -4, -4, -4, -4, -4, -4, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1],
    [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0],
    [0, -4, 4, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0],
    [0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1],
    [0, 0, 0, -4, 4, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1],
    [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1],
    [0, 0, 0, 0, 0, -4, 4, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1],
    [0, 2, 2, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2],
    [0, -4, -4, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2],
    [0, 0, 0, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0],
    [0, 0, 0, -2, -2, 2, 2, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0],
    [0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 0, 0, 0, 0],
    [0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1],
    [0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0],
    [0, 0, 0, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, -1, 1, 0, 0, 0, 0],
    [0, 0, 0, 0, 0, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, 1, -1, 1, -1],
    [0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1, -1, -1, 1, 1]], dtype=np.float64)
CONSERVED = [0, 3, 5, 7]  # moment rows of mass and momentum
# stress components in the order xx, yy, zz, xy, xz, yz
PAIRS = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))


def bf16(x):
    """Round FP32 values to BFloat16 (round to nearest, ties to even), returned as FP32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    lsb = (b >> np.uint64(16)) & np.uint64(1)
    r = ((b + np.uint64(0x7FFF) + lsb) >> np.uint64(16)) << np.uint64(16)
    out = (r & np.uint64(0xFFFFFFFF)).astype(np.uint32).view(np.float32)
    nan = np.isnan(a)
    if nan.any():
        out = out.copy()
        out[nan] = np.nan
    return out.reshape(np.shape(x))


def gelu(z):
    """Tanh-form GELU (Hendrycks and Gimpel, 2016): 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))."""
    z = np.asarray(z, dtype=np.float64)
    return 0.5 * z * (1.0 + np.tanh(GELU_K * (z + GELU_A * z ** 3)))


A_BF16 = 0.044677734375   # 0.044715 rounded to BFloat16
K_BF16 = 0.796875         # sqrt(2 / pi) rounded to BFloat16


def gelu_bf16(z):
    """The device's inference GELU on BF16 pairs: z^2, fma(z^2, a, 1), k z, k z (1 + a z^2), tanh,
    z / 2, fma(z / 2, t, z / 2), each result rounded to BF16 (tanh by numpy in place of the hardware
    approximation)."""
    r = lambda v: bf16(np.asarray(v, np.float64).astype(np.float32)).astype(np.float64)
    zb = r(z)
    p = r(r(zb * zb) * A_BF16 + 1.0)
    arg = r(r(zb * K_BF16) * p)
    t = r(np.tanh(arg))
    hz = r(zb * 0.5)
    return r(hz * t + hz)


def gelu_grad(z):
    z = np.asarray(z, dtype=np.float64)
    t = np.tanh(GELU_K * (z + GELU_A * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_K * (1.0 + 3.0 * GELU_A * z * z)


# ---------------------------------------------------------------- features
def feq19(rho, u):
    """Second-order equilibrium (lbm_solver_interface.cpp:374-435), rho [n], u [n, 3] -> [n, 19]."""
    cu = u @ C19.T
    uu = (u * u).sum(axis=1, keepdims=True)
    return W19 * rho[:, None] * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * uu)


def macros19(f):
    rho = f.sum(axis=1)
    return rho, (f @ C19) / rho[:, None]


def stress(neq):
    """Pi_ab = sum_q c_a c_b neq_q, [n, 6] in the order xx, yy, zz, xy, xz, yz."""
    return np.stack([(neq * (C19[:, a] * C19[:, b])).sum(axis=1) for a, b in PAIRS], axis=1)


def double_dot(a, b):
    """A:B of symmetric tensors stored as [n, 6]."""
    return (a[:, :3] * b[:, :3]).sum(axis=1) + 2.0 * (a[:, 3:] * b[:, 3:]).sum(axis=1)


def smagorinsky_increment(pi, tau0, c):
    """tau_sgs = 0.5 (sqrt(tau0^2 + 18 c sqrt(2 Pi:Pi)) - tau0) (lbm_les_smagorinsky.cpp:22-94 with C = 18 c)."""
    return 0.5 * (np.sqrt(tau0 * tau0 + 18.0 * c * np.sqrt(2.0 * double_dot(pi, pi))) - tau0)


def features(rho, neq, tau0):
    """The 24 network inputs of a node: the 19 non-equilibrium MRT moments / rho (the conserved
    four set to zero) and five
    invariants of the strain estimate S = -3 Pi / (2 rho tau0): tr S, S:S, tr(Sd^3), |Sd| and the
    Smagorinsky (Cs = 0.1) increment of tau."""
    rho = np.asarray(rho, dtype=np.float64)
    m = (neq @ M19.T) / rho[:, None]
    m[:, CONSERVED] = 0.0  # mass and momentum of f - feq vanish: exact zero inputs
    pi = stress(neq)
    s = -1.5 / (rho * tau0)[:, None] * pi if np.ndim(tau0) else -1.5 / (rho[:, None] * tau0) * pi
    tr = s[:, 0] + s[:, 1] + s[:, 2]
    sd = s.copy()
    sd[:, :3] -= tr[:, None] / 3.0
    ss = double_dot(s, s)
    a, b, c, d, e, g = (sd[:, i] for i in range(6))  # xx yy zz xy xz yz
    det = a * (b * c - g * g) - d * (d * c - g * e) + e * (d * g - b * e)
    inv3 = 3.0 * det
    mag = np.sqrt(2.0 * double_dot(sd, sd))
    smag = smagorinsky_increment(pi, tau0, C_UNIT)
    return np.concatenate([m, np.stack([tr, ss, inv3, mag, smag], axis=1)], axis=1)


def node_features(f, tau0):
    """Features of nodes given their (post-stream) populations f [n, 19]."""
    f = np.asarray(f, dtype=np.float64)
    rho, u = macros19(f)
    return features(rho, f - feq19(rho, u), tau0)


# ---------------------------------------------------------------- network
class Mlp:
    """Weights of the closure network; arrays are FP32 like the device's master copy."""

    def __init__(self, w1, b1, w2, b2, w3, b3, mean, inv_std):
        self.w1 = np.asarray(w1, np.float32).reshape(N_HID, N_IN)
        self.b1 = np.asarray(b1, np.float32).reshape(N_HID)
        self.w2 = np.asarray(w2, np.float32).reshape(N_HID, N_HID)
        self.b2 = np.asarray(b2, np.float32).reshape(N_HID)
        self.w3 = np.asarray(w3, np.float32).reshape(N_HID)
        self.b3 = np.float32(b3)
        self.mean = np.asarray(mean, np.float32).reshape(N_IN)
        self.inv_std = np.asarray(inv_std, np.float32).reshape(N_IN)

    @staticmethod
    def random(seed: int, mean=None, inv_std=None):
        rng = np.random.default_rng(seed)
        w1 = rng.normal(0, np.sqrt(2.0 / N_IN), (N_HID, N_IN))
        w2 = rng.normal(0, np.sqrt(2.0 / N_HID), (N_HID, N_HID))
        w3 = rng.normal(0, np.sqrt(1.0 / N_HID), N_HID)
        return Mlp(w1, rng.normal(0, 0.1, N_HID), w2, rng.normal(0, 0.1, N_HID), w3, 1.0,
                   np.zeros(N_IN) if mean is None else mean, np.ones(N_IN) if inv_std is None else inv_std)

    def flat(self):
        """Parameters in the order of zl_mlp: w1, b1, w2, b2, w3, b3, in_mean, in_inv_std."""
        return np.concatenate([self.w1.ravel(), self.b1, self.w2.ravel(), self.b2, self.w3, [self.b3],
                               self.mean, self.inv_std]).astype(np.float32)

    @staticmethod
    def from_flat(v):
        v = np.asarray(v, np.float32)
        o = 0
        parts = []
        for size in (N_HID * N_IN, N_HID, N_HID * N_HID, N_HID, N_HID, 1, N_IN, N_IN):
            parts.append(v[o:o + size])
            o += size
        return Mlp(parts[0], parts[1], parts[2], parts[3], parts[4], parts[5][0], parts[6], parts[7])

    # forward with the device's rounding points (rounding=False: plain FP64, for finite-difference
    # checks of the backward formulas); returns y and the intermediates of backward
    def forward(self, x, rounding: bool = True, inference: bool = False):
        """inference=True: the GELU of the device's inference kernels (gelu_bf16)."""
        r = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
        x = np.asarray(x, np.float32 if rounding else np.float64)
        xh = np.asarray(r((x - self.mean) * self.inv_std), np.float64)
        z1 = xh @ np.asarray(r(self.w1), np.float64).T + np.asarray(r(self.b1), np.float64)
        if inference:
            a1 = gelu_bf16(z1)
        else:
            a1 = np.asarray(r(gelu(z1).astype(np.float32) if rounding else gelu(z1)), np.float64)
        z2 = a1 @ np.asarray(r(self.w2), np.float64).T + np.asarray(r(self.b2), np.float64)
        a2 = gelu_bf16(z2) if inference else gelu(z2)
        y = a2 @ self.w3.astype(np.float64) + float(self.b3)
        return y, (xh, z1, a1, z2, a2)

    def predict_c(self, x, fallback_c=C_UNIT):
        y, _ = self.forward(x, inference=True)
        c = C_UNIT * np.clip(y, 0.0, Y_MAX)
        return np.where(np.isfinite(y), c, fallback_c)

    def gradients(self, x, t, rounding: bool = True):
        """Mean-square-error loss and its gradients (dict of arrays shaped like the weights)."""
        r = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
        y, (xh, z1, a1, z2, a2) = self.forward(x, rounding)
        n = y.shape[0]
        err = y - np.asarray(t, np.float64)
        loss = float((err * err).mean())
        dy = 2.0 * err / n
        g = {"w3": a2.T @ dy, "b3": dy.sum()}
        dz2 = (dy[:, None] * self.w3.astype(np.float64)) * gelu_grad(z2)
        dz2b = np.asarray(r(dz2.astype(np.float32) if rounding else dz2), np.float64)
        g["b2"] = dz2b.sum(axis=0)  # a ones column of the tensor-core product
        g["w2"] = dz2b.T @ a1
        da1 = dz2b @ np.asarray(r(self.w2), np.float64)
        dz1 = da1 * gelu_grad(z1)
        dz1b = np.asarray(r(dz1.astype(np.float32) if rounding else dz1), np.float64)
        g["b1"] = dz1b.sum(axis=0)
        g["w1"] = dz1b.T @ xh
        return loss, g


class Adam:
    """Adam (Kingma and Ba, 2015) with bias correction, FP32 moments, like the device trainer."""

    def __init__(self, net: Mlp, b1=0.9, b2=0.999, eps=1e-8):
        self.net, self.b1, self.b2, self.eps, self.t = net, b1, b2, eps, 0
        self.m = {k: np.zeros_like(getattr(net, k), dtype=np.float64) for k in ("w1", "b1", "w2", "b2", "w3", "b3")}
        self.v = {k: np.zeros_like(self.m[k]) for k in self.m}

    def step(self, grads, lr):
        self.t += 1
        for k in self.m:
            g = np.asarray(grads[k], np.float64)
            self.m[k] = self.b1 * self.m[k] + (1 - self.b1) * g
            self.v[k] = self.b2 * self.v[k] + (1 - self.b2) * g * g
            mh = self.m[k] / (1 - self.b1 ** self.t)
            vh = self.v[k] / (1 - self.b2 ** self.t)
            new = np.asarray(getattr(self.net, k), np.float64) - lr * mh / (np.sqrt(vh) + self.eps)
            setattr(self.net, k, np.float32(new) if k == "b3" else new.astype(np.float32))


def learned_tau(pi, tau0, c):
    return tau0 + smagorinsky_increment(pi, tau0, c)


# ---------------------------------------------------------------- filter and training pairs
def box_filter(f_fine, n_fine, factor):
    """Box filter of fine populations f [nx*ny*nz, 19] (x fastest) over factor^3 blocks.
    Returns [n_coarse, 29]: rho, u (3), <u_a u_b> (6, xx yy zz xy xz yz), <neq> (19), block means."""
    nx, ny, nz = n_fine
    f = np.asarray(f_fine, np.float64)
    rho, u = macros19(f)
    neq = f - feq19(rho, u)
    uu = np.stack([u[:, a] * u[:, b] for a, b in PAIRS], axis=1)
    fields = np.concatenate([rho[:, None], u, uu, neq], axis=1)  # [n, 29]
    g = fields.reshape(nz // factor, factor, ny // factor, factor, nx // factor, factor, 29)
    return g.mean(axis=(1, 3, 5)).reshape(-1, 29)


def filtered_strain(rho, neq, tau_fine, factor):
    """Strain of the filtered field in coarse lattice units, S = -3 factor Pi<f - feq> / (2 rho tau_f):
    the fine non-equilibrium stress is -2/3 rho tau_f S_fine and S_coarse = factor S_fine."""
    return -1.5 * factor / (rho * tau_fine)[:, None] * stress(neq)


def box3_mean(v, n):
    """Mean over the 3x3x3 neighbourhood on a periodic grid."""
    nx, ny, nz = n
    g = v.reshape(nz, ny, nx)
    acc = np.zeros_like(g)
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                acc += np.roll(g, (dz, dy, dx), axis=(0, 1, 2))
    return (acc / 27.0).ravel()


def training_pairs(filtered, n_coarse, tau_fine, tau_coarse, factor):
    """Features and targets y = c / 0.01 of every coarse node from the filtered fine fields.

    Target: least-squares Smagorinsky coefficient of the exact subgrid stress
    tau_ab = <u_a u_b> - <u_a><u_b> over the 3x3x3 neighbourhood,
    c = -<tau^d : M> / <M : M> with M = 2 |S| S, clipped to [0, 8 * 0.01]; S is the strain of the
    filtered field as the coarse collision estimates it, from the filtered non-equilibrium stress.
    Features: those of a coarse node whose populations are feq(<rho>, <u>) plus the filtered
    non-equilibrium part rescaled to the coarse step, r <neq> with r = factor * tau_eff / tau_fine
    and tau_eff = tau_coarse + 3 c |S| (the relaxation time that node runs with)."""
    rho, u, uu, neq = filtered[:, 0], filtered[:, 1:4], filtered[:, 4:10], filtered[:, 10:29]
    s = filtered_strain(rho, neq, tau_fine, factor)
    smag = np.sqrt(2.0 * double_dot(s, s))
    tau_sgs = uu - np.stack([u[:, a] * u[:, b] for a, b in PAIRS], axis=1)
    trace = tau_sgs[:, :3].sum(axis=1)
    tau_d = tau_sgs.copy()
    tau_d[:, :3] -= trace[:, None] / 3.0
    mm = 2.0 * smag[:, None] * s
    num = box3_mean(double_dot(tau_d, mm), n_coarse)
    den = box3_mean(double_dot(mm, mm), n_coarse)
    ok = den > DEN_MIN  # no resolved strain: no model constant to fit
    c = np.where(ok, -num / np.where(ok, den, 1.0), 0.0)
    y = np.clip(c / C_UNIT, 0.0, Y_MAX)
    tau_eff = tau_coarse + 3.0 * C_UNIT * y * smag
    r = factor * tau_eff / tau_fine
    x = features(rho, r[:, None] * neq, tau_coarse)
    return x.astype(np.float32), y.astype(np.float32)


def energy_spectrum(u, n):
    """Shell-summed kinetic-energy spectrum E(k), k = 0 .. n/2, of a periodic cubic field u [n^3, 3]."""
    g = np.asarray(u, np.float64).reshape(n, n, n, 3)
    uh = np.fft.fftn(g, axes=(0, 1, 2)) / n ** 3
    e = 0.5 * (np.abs(uh) ** 2).sum(axis=-1)
    k = np.fft.fftfreq(n, 1.0 / n)
    kk = np.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2)
    shell = np.rint(kk).astype(np.int64)
    out = np.bincount(shell.ravel(), weights=e.ravel(), minlength=n)
    return out[: n // 2 + 1]
