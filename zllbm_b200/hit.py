"""Learned LES closure on decaying homogeneous isotropic turbulence (HIT).

Workload: a fine D3Q19 SRT run on an N^3 periodic box, box-filtered by `factor` to the coarse
grid, supplies training pairs (node features -> least-squares Smagorinsky constant of the exact
subgrid stress); the closure network is trained on the GPU by the library's tensor-core trainer;
then coarse runs with Smagorinsky (Cs = 0.1) and with the learned closure start from the filtered
initial field and are compared with the filtered fine run through their kinetic-energy spectra.

Initial field: random-phase solenoidal Fourier modes with E(k) ~ k^4 exp(-2 (k / k0)^2), scaled
to u_rms, rho = 1, populations at equilibrium (seeded; the reference has no HIT case).
Scaling between the grids is acoustic: dx_c = factor dx_f, dt_c = factor dt_f, so the lattice
viscosity is nu_c = nu_f / factor and velocities are the same in both lattice units.

Device memory and the spectra's FFTs use torch; every lattice update, filter, feature, training
and inference kernel is the library's (libzllbm_b200.so through the C ABI).
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

import zllbm_b200 as zl


def hit_velocity(n: int, k0: float = 4.0, u_rms: float = 0.04, seed: int = 20261203):
    """Solenoidal random-phase velocity on an n^3 periodic grid (torch CUDA tensor [n^3, 3], FP32)."""
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    k = torch.fft.fftfreq(n, 1.0 / n, device="cuda")
    kr = torch.fft.rfftfreq(n, 1.0 / n, device="cuda")
    kz, ky, kx = torch.meshgrid(k, k, kr, indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    kk = torch.sqrt(k2)
    # shell energy E(k) ~ k^4 exp(-2 (k/k0)^2) spread over the shell's ~4 pi k^2 modes
    amp = torch.where(kk > 0, torch.sqrt(kk ** 4 * torch.exp(-2.0 * (kk / k0) ** 2) / (4 * math.pi * k2.clamp(min=1))),
                      torch.zeros_like(kk))
    comps = []
    for _ in range(3):
        re = torch.randn(kk.shape, generator=g, device="cuda")
        im = torch.randn(kk.shape, generator=g, device="cuda")
        comps.append(torch.complex(re, im) * amp)
    ax, ay, az = comps
    # project out the compressive part: a - k (k . a) / |k|^2
    kd = (kx * ax + ky * ay + kz * az) / k2.clamp(min=1)
    ax, ay, az = ax - kx * kd, ay - ky * kd, az - kz * kd
    u = torch.stack([torch.fft.irfftn(c, s=(n, n, n)) for c in (ax, ay, az)], dim=-1)  # [z, y, x, 3]
    u = u * (u_rms / torch.sqrt((u * u).sum(dim=-1).mean() / 3.0))
    return u.reshape(-1, 3).float().contiguous()


def energy_spectrum(u, n: int) -> np.ndarray:
    """Shell-summed kinetic energy E(k), k = 0 .. n/2 (rounded |k|), of u [n^3, 3] (x fastest)."""
    import torch
    g = u.reshape(n, n, n, 3).double()
    uh = torch.fft.fftn(g, dim=(0, 1, 2)) / n ** 3
    e = 0.5 * (uh.real ** 2 + uh.imag ** 2).sum(dim=-1)
    k = torch.fft.fftfreq(n, 1.0 / n, device=u.device).double()
    kk = torch.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2)
    shell = torch.round(kk).long().reshape(-1)
    out = torch.zeros(int(shell.max()) + 1, dtype=torch.float64, device=u.device)
    out.index_add_(0, shell, e.reshape(-1))
    return out[: n // 2 + 1].cpu().numpy()


def spectrum_error(e_model: np.ndarray, e_ref: np.ndarray, k_max: int) -> float:
    """Root-mean-square of log(E_model / E_ref) over shells 1 .. k_max."""
    a, b = e_model[1:k_max + 1], e_ref[1:k_max + 1]
    return float(np.sqrt(np.mean(np.log(np.maximum(a, 1e-300) / np.maximum(b, 1e-300)) ** 2)))


def box_context(n: int, tau: float, storage: int = zl.STORAGE_F32, les: int = zl.LES_OFF, cs: float = 0.0,
                collision: int = zl.SRT, device: int = 0, rounding: int = zl.ROUND_STOCHASTIC) -> zl.Context:
    """A full periodic n^3 box level issuing on torch's current stream (so that torch work on the
    fields and the library's kernels stay ordered; that stream must not be the legacy default one)."""
    import torch
    cfg = zl.SolverConfig(lattice=zl.D3Q19, collision=collision, storage=storage, viscosity=(tau - 0.5) / 3.0,
                          bc_kind=(zl.BC_PERIODIC,) * 6, domain_min=(0, 0, 0), domain_max=(n, n, n), les=les,
                          les_cs=cs, device=device, storage_rounding=rounding)
    ctx = zl.Context(cfg)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream or None)
    ctx.set_level_box(0, (0, 0, 0), (n, n, n))
    return ctx


@dataclass
class HitConfig:
    fine: int = 1024           # fine lattice edge
    factor: int = 4            # filter width = coarse spacing in fine cells
    nu_fine: float = 0.002     # fine lattice viscosity
    k0: float = 4.0
    u_rms: float = 0.04
    seed: int = 20261203
    coarse_steps: int = 10000
    checkpoints: int = 10      # spectra compared at this many evenly spaced coarse times
    train_snapshots: int = 4   # filtered fine snapshots used as training data (first half of the run)
    train_steps: int = 2000    # Adam steps (mini-batches drawn without replacement, epoch after epoch)
    batch: int = 128 * 148 * 2
    lr: float = 2e-3           # cosine-decayed to lr / 20
    closure_every: int = 8     # the amortised variant evaluates the network on every k-th step
    # network output scales and Smagorinsky constants tried by the calibration (both searches
    # reach well below the optima seen so far, alpha 0.3 - 0.5 and Cs 0.06 - 0.08)
    calibrate_alpha: tuple = (0.05, 0.1, 0.15, 0.2, 0.25, 0.3, 0.4, 0.5, 0.6, 0.8, 1.0)
    calibrate_cs: tuple = (0.02, 0.03, 0.04, 0.05, 0.06, 0.07, 0.08, 0.09, 0.1, 0.12)
    test_realizations: int = 3  # independent test fields (seeds seed + 1000 k, k = 1 ..)
    storage: int = zl.STORAGE_F32
    fine_storage: int = zl.STORAGE_F32
    cs: float = 0.1

    @property
    def coarse(self) -> int:
        return self.fine // self.factor

    @property
    def tau_fine(self) -> float:
        return 0.5 + 3.0 * self.nu_fine

    @property
    def tau_coarse(self) -> float:
        return 0.5 + 3.0 * self.nu_fine / self.factor


@dataclass
class HitResult:
    config: dict
    times: list = field(default_factory=list)
    spectra: dict = field(default_factory=dict)
    errors: dict = field(default_factory=dict)
    mlups: dict = field(default_factory=dict)
    training: dict = field(default_factory=dict)


def _filtered_velocity(ctx, cfg: HitConfig, buf):
    import torch
    ctx.filter_level(0, cfg.factor, buf.data_ptr())
    ctx.synchronize()
    return buf[:, 1:4].contiguous(), buf[:, 0].contiguous()


def initial_net(seed: int, in_mean=None, in_inv_std=None) -> "zl.ZlMlp":
    """He-initialised closure network (zero hidden biases, output bias 1 = the Smagorinsky value)
    with the given input normalisation (identity when omitted)."""
    rng = np.random.default_rng(seed)
    w1 = rng.normal(0, math.sqrt(2.0 / 24), (64, 24))
    w2 = rng.normal(0, math.sqrt(2.0 / 64), (64, 64))
    w3 = rng.normal(0, 0.1 * math.sqrt(1.0 / 64), 64)
    mean = np.zeros(24) if in_mean is None else np.asarray(in_mean)
    inv = np.ones(24) if in_inv_std is None else np.asarray(in_inv_std)
    flat = np.concatenate([w1.ravel(), np.zeros(64), w2.ravel(), np.zeros(64), w3, [1.0], mean, inv])
    return zl.ZlMlp.from_flat(flat.astype(np.float32))


def train(x, y, cfg: HitConfig, log=print):
    """Train the closure network on device tensors x [n, 24], y [n] with the library's trainer.
    Returns the ZlMlp and a dict of losses (train, held-out, constant Smagorinsky y = 1)."""
    import torch
    n = x.shape[0]
    g = torch.Generator(device="cuda")
    g.manual_seed(cfg.seed + 1)
    perm = torch.randperm(n, generator=g, device="cuda")
    n_val = max(1, n // 20)
    val, tr_idx = perm[:n_val], perm[n_val:]
    mean = x[tr_idx].mean(dim=0)
    std = x[tr_idx].std(dim=0)
    inv = torch.where(std > 0, 1.0 / std.clamp(min=1e-30), torch.ones_like(std))
    net = initial_net(cfg.seed + 2, mean.cpu().numpy(), inv.cpu().numpy())
    xv, yv = x[val].contiguous(), y[val].contiguous()
    yp = torch.empty_like(yv)

    def val_loss(m):
        zl.mlp_forward(m, xv.data_ptr(), xv.shape[0], yp.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        return float(((yp - yv) ** 2).mean())

    history = []
    t0 = time.perf_counter()
    steps, epoch = 0, 0
    batch = min(cfg.batch, tr_idx.numel())
    report = max(1, cfg.train_steps // 10)
    with zl.Trainer(net) as trainer:
        trainer.set_stream(torch.cuda.current_stream().cuda_stream)
        while steps < cfg.train_steps:
            order = tr_idx[torch.randperm(tr_idx.numel(), generator=g, device="cuda")]
            for s in range(0, order.numel() - batch + 1, batch):
                idx = order[s:s + batch]
                lr = cfg.lr * (0.05 + 0.95 * 0.5 * (1.0 + math.cos(math.pi * steps / cfg.train_steps)))
                xb, yb = x[idx].contiguous(), y[idx].contiguous()
                trainer.step(xb.data_ptr(), yb.data_ptr(), idx.numel(), lr)
                steps += 1
                if steps % report == 0 or steps == cfg.train_steps:
                    loss = trainer.loss()
                    vl = val_loss(trainer.weights())
                    history.append({"step": steps, "epoch": epoch, "batch_loss": loss, "val_loss": vl})
                    log(f"step {steps} (epoch {epoch}): batch loss {loss:.4g}, held-out loss {vl:.4g}")
                if steps >= cfg.train_steps:
                    break
            epoch += 1
        net = trainer.weights()
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    const_smag = float(((yv - 1.0) ** 2).mean())
    const_best = float(((yv - y[tr_idx].mean()) ** 2).mean())
    vl = val_loss(net)
    return net, {"history": history, "val_loss": vl, "val_loss_smagorinsky_y1": const_smag,
                 "val_loss_best_constant": const_best, "samples": int(n), "steps": steps, "epochs": epoch,
                 "batch": batch, "seconds": train_s, "target_mean": float(y.mean()), "target_std": float(y.std()),
                 "val_prediction_mean": float(yp.mean()), "val_prediction_std": float(yp.std())}


def predicted_y(ctx, net, n: int):
    """Mean and standard deviation of the network output over a coarse level's nodes."""
    import torch
    x = torch.empty((n ** 3, 24), dtype=torch.float32, device="cuda")
    yv = torch.empty(n ** 3, dtype=torch.float32, device="cuda")
    ctx.closure_features(0, x.data_ptr())
    zl.mlp_forward(net, x.data_ptr(), n ** 3, yv.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return float(yv.mean()), float(yv.std())


def _time_steps(ctx, steps: int) -> float:
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.synchronize()
    a.record(stream)
    for _ in range(steps):
        ctx.step_level(0)
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b)


def closure_cost(net, n: int, tau: float, intervals=(1, 8, 16), steps: int = 96, cs: float = 0.1,
                 seed: int = 1) -> dict:
    """MLUPS of the coarse step on an n^3 HIT box with Smagorinsky and with the network evaluated on
    every k-th step for each k in `intervals` (kernel time, CUDA events, after warm-up)."""
    import torch
    u = hit_velocity(n, seed=seed)
    rho = torch.ones(n ** 3, dtype=torch.float32, device="cuda")
    out = {"grid": n, "steps": steps}
    variants = [("smagorinsky", zl.LES_SMAGORINSKY, 1)]
    variants += [("learned" if k == 1 else f"learned_every{k}", zl.LES_LEARNED, k) for k in intervals]
    for name, les, k in variants:
        ctx = box_context(n, tau, les=les, cs=cs)
        if les == zl.LES_LEARNED:
            ctx.set_closure(net)
            ctx.set_closure_interval(k)
        ctx.set_equilibrium_dense(0, rho.data_ptr(), u.data_ptr())
        _time_steps(ctx, 2 * k + 4)
        ms = _time_steps(ctx, steps)
        out[name] = float(n) ** 3 * steps / (ms / 1e3) / 1e6
        ctx.close()
    for name, _, _ in variants[1:]:
        out[f"{name}_cost_fraction"] = 1.0 - out[name] / out["smagorinsky"]
    return out


def run(cfg: HitConfig, log=print) -> HitResult:
    """The whole case on one non-default stream (torch, contexts and trainer share it)."""
    import torch
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        res = _run(cfg, log)
    stream.synchronize()
    return res


@dataclass
class FineReference:
    spectra: dict            # coarse step -> filtered fine spectrum
    rho0: object             # filtered initial density / velocity (coarse grid)
    u0: object
    pairs: tuple = ()        # (x, y) device tensors of the training snapshots
    mlups: float = 0.0
    seconds: float = 0.0


def fine_reference(cfg: HitConfig, seed: int, ck_times, snap_times=(), log=print) -> FineReference:
    """Fine run of one realization: filtered spectra at ck_times (coarse steps) and training pairs
    at snap_times."""
    import torch
    nf, nc, fac = cfg.fine, cfg.coarse, cfg.factor
    u0 = hit_velocity(nf, cfg.k0, cfg.u_rms, seed)
    torch.cuda.empty_cache()  # the FFT work space goes back before the populations are allocated
    fine = box_context(nf, cfg.tau_fine, storage=cfg.fine_storage)
    rho0 = torch.ones(nf ** 3, dtype=torch.float32, device="cuda")
    fine.set_equilibrium_dense(0, rho0.data_ptr(), u0.data_ptr())
    fine.synchronize()
    del u0, rho0
    torch.cuda.empty_cache()
    filt = torch.empty((nc ** 3, 29), dtype=torch.float32, device="cuda")
    u_bar0, rho_bar0 = _filtered_velocity(fine, cfg, filt)
    ref = FineReference(spectra={}, rho0=rho_bar0.clone(), u0=u_bar0.clone())
    xs, ys = [], []
    scratch = torch.empty((nc ** 3, 3), dtype=torch.float32, device="cuda")
    t0 = time.perf_counter()
    ms, t = 0.0, 0
    for target in sorted(set(ck_times) | set(snap_times)):
        if target > t:
            ms += _time_steps(fine, (target - t) * fac)
            t = target
        u_bar, _ = _filtered_velocity(fine, cfg, filt)
        if t in ck_times:
            ref.spectra[t] = energy_spectrum(u_bar, nc)
        if t in snap_times:
            x = torch.empty((nc ** 3, 24), dtype=torch.float32, device="cuda")
            y = torch.empty(nc ** 3, dtype=torch.float32, device="cuda")
            zl.closure_pairs((nc, nc, nc), filt.data_ptr(), cfg.tau_fine, cfg.tau_coarse, fac, x.data_ptr(),
                             y.data_ptr(), scratch.data_ptr(), torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            xs.append(x)
            ys.append(y)
        log(f"seed {seed}, fine step {t * fac}")
    fine.close()
    del fine
    torch.cuda.empty_cache()
    ref.mlups = float(nf) ** 3 * t * fac / (ms / 1e3) / 1e6 if ms > 0 else 0.0
    ref.seconds = time.perf_counter() - t0
    if xs:
        ref.pairs = (torch.cat(xs), torch.cat(ys))
    return ref


def scaled_net(net: "zl.ZlMlp", alpha: float) -> "zl.ZlMlp":
    """The network with its output scaled by alpha (w3, b3 times alpha): c = alpha * c_network."""
    v = net.flat().copy()
    o_w3 = 64 * 24 + 64 + 64 * 64 + 64
    v[o_w3:o_w3 + 65] *= alpha
    return zl.ZlMlp.from_flat(v)


def coarse_run(cfg: HitConfig, ref: FineReference, ck_times, les: int, cs: float, net=None, every: int = 1,
               diagnose: bool = False):
    """One coarse LES run from the filtered initial field; spectra and errors against `ref`."""
    import torch
    nc = cfg.coarse
    ctx = box_context(nc, cfg.tau_coarse, storage=cfg.storage, les=les, cs=cs)
    if les == zl.LES_LEARNED:
        ctx.set_closure(net)
        ctx.set_closure_interval(every)
    ctx.set_equilibrium_dense(0, ref.rho0.data_ptr(), ref.u0.data_ptr())
    rho_d = torch.empty(nc ** 3, dtype=torch.float32, device="cuda")
    u_d = torch.empty((nc ** 3, 3), dtype=torch.float32, device="cuda")
    spectra, errs, errs_low, pred = {}, [], [], []
    t, ms = 0, 0.0
    for target in ck_times:
        if target > t:
            ms += _time_steps(ctx, target - t)
            t = target
        ctx.get_macros_dense(0, rho_d.data_ptr(), u_d.data_ptr())
        ctx.synchronize()
        e = energy_spectrum(u_d, nc)
        spectra[str(t)] = e.tolist()
        if t > 0:
            if diagnose and net is not None:
                pred.append(predicted_y(ctx, net, nc))
            errs.append(spectrum_error(e, ref.spectra[t], nc // 2 - 1))
            errs_low.append(spectrum_error(e, ref.spectra[t], nc // 4))
        if not np.all(np.isfinite(e)):
            errs.append(float("inf"))
            errs_low.append(float("inf"))
            break
    ctx.close()
    return {"error": float(np.mean(errs)) if errs else None, "error_k_le_n/4": float(np.mean(errs_low)) if errs_low else None,
            "per_checkpoint": errs, "spectra": spectra, "mlups": float(nc) ** 3 * t / (ms / 1e3) / 1e6 if ms else None,
            "predicted_y": pred}


def _run(cfg: HitConfig, log=print) -> HitResult:
    """Training realization (seed): fine run, training pairs, network training, and a one-number
    calibration of the network output scale (and, for a fair comparison, of the Smagorinsky
    constant) against its filtered spectra.  Test realizations (seeds seed + 1000 k): fresh fine
    runs against which Smagorinsky (configured and calibrated constant) and the learned closure
    (raw and calibrated) are scored; errors are the mean over realizations with their spread."""
    import torch
    res = HitResult(config={**cfg.__dict__, "coarse": cfg.coarse, "tau_fine": cfg.tau_fine,
                            "tau_coarse": cfg.tau_coarse})
    nc = cfg.coarse
    every = max(1, cfg.coarse_steps // cfg.checkpoints)
    ck_times = [every * i for i in range(cfg.checkpoints + 1)]
    snap_times = [int(cfg.coarse_steps / 2 * (i + 1) / cfg.train_snapshots) for i in range(cfg.train_snapshots)]
    res.times = ck_times

    train_ref = fine_reference(cfg, cfg.seed, ck_times, snap_times, log)
    res.mlups["fine_srt"] = train_ref.mlups
    x, y = train_ref.pairs
    train_ref.pairs = ()
    net, info = train(x, y, cfg, log)
    res.training.update(info)
    del x, y
    torch.cuda.empty_cache()

    # calibration on the training realization
    calib = {"alpha": {}, "cs": {}}
    for a in cfg.calibrate_alpha:
        r = coarse_run(cfg, train_ref, ck_times, zl.LES_LEARNED, cfg.cs, scaled_net(net, a), cfg.closure_every)
        calib["alpha"][f"{a:g}"] = r["error"]
        log(f"calibration: alpha {a:g} -> {r['error']}")
    for c in cfg.calibrate_cs:
        r = coarse_run(cfg, train_ref, ck_times, zl.LES_SMAGORINSKY, c)
        calib["cs"][f"{c:g}"] = r["error"]
        log(f"calibration: Cs {c:g} -> {r['error']}")
    finite = lambda d: {k: v for k, v in d.items() if v is not None and np.isfinite(v)}
    alpha = float(min(finite(calib["alpha"]).items(), key=lambda kv: kv[1])[0]) if finite(calib["alpha"]) else 1.0
    cs_best = float(min(finite(calib["cs"]).items(), key=lambda kv: kv[1])[0]) if finite(calib["cs"]) else cfg.cs
    res.training["calibration"] = {**calib, "alpha_best": alpha, "cs_best": cs_best}
    del train_ref
    torch.cuda.empty_cache()

    # evaluation on independent realizations: every model scored on each, mean and spread reported
    net_cal = scaled_net(net, alpha)
    runs = [("smagorinsky", zl.LES_SMAGORINSKY, cfg.cs, None, 1),
            (f"smagorinsky_calibrated", zl.LES_SMAGORINSKY, cs_best, None, 1),
            ("learned", zl.LES_LEARNED, cfg.cs, net, 1),
            ("learned_calibrated", zl.LES_LEARNED, cfg.cs, net_cal, 1),
            (f"learned_calibrated_every{cfg.closure_every}", zl.LES_LEARNED, cfg.cs, net_cal, cfg.closure_every)]
    res.training["coarse_predicted_y"] = {}
    per = {name: [] for name, *_ in runs}
    for t in range(max(1, cfg.test_realizations)):
        seed = cfg.seed + 1000 * (t + 1)
        test_ref = fine_reference(cfg, seed, ck_times, (), log)
        if t == 0:
            res.spectra["filtered_fine"] = {str(k): v.tolist() for k, v in test_ref.spectra.items()}
        for name, les, cs, n_, k in runs:
            r = coarse_run(cfg, test_ref, ck_times, les, cs, n_, k, diagnose=n_ is not None and t == 0)
            spectra, pred, mlups = r.pop("spectra"), r.pop("predicted_y"), r.pop("mlups")
            if t == 0:
                res.spectra[name] = spectra
                res.training["coarse_predicted_y"][name] = pred
                res.mlups[name] = mlups
            per[name].append({"seed": seed, **r})
            log(f"{name} (seed {seed}): spectrum error {r['error']} (k <= n/4: {r['error_k_le_n/4']})")
        del test_ref
        torch.cuda.empty_cache()
    for name, rs in per.items():
        # a run without a finite spectrum (unstable) scores infinity
        errs = np.array([np.inf if r["error"] is None else r["error"] for r in rs], dtype=np.float64)
        low = np.array([np.inf if r["error_k_le_n/4"] is None else r["error_k_le_n/4"] for r in rs], dtype=np.float64)
        res.errors[name] = {"error": float(errs.mean()), "error_std": float(errs.std(ddof=1)) if errs.size > 1 else 0.0,
                            "error_k_le_n/4": float(low.mean()), "per_realization": rs}
    # the learned closure against Smagorinsky calibrated the same way, realization by realization
    diff = np.array([(np.inf if a["error"] is None else a["error"]) - (np.inf if b["error"] is None else b["error"])
                     for a, b in zip(per["learned_calibrated"], per["smagorinsky_calibrated"])])
    res.errors["learned_minus_smagorinsky_calibrated"] = {"mean": float(diff.mean()),
                                                          "std": float(diff.std(ddof=1)) if diff.size > 1 else 0.0,
                                                          "per_realization": diff.tolist()}
    res.mlups["cost"] = closure_cost(net_cal, max(256, nc), cfg.tau_coarse, (1, 8, 16, cfg.closure_every))
    log(f"closure cost on {max(256, nc)}^3: {res.mlups['cost']}")
    res.training["net"] = net.flat().tolist()
    res.training["alpha"] = alpha
    return res


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="learned LES closure on decaying HIT")
    ap.add_argument("--fine", type=int, default=1024)
    ap.add_argument("--factor", type=int, default=4)
    ap.add_argument("--nu", type=float, default=0.002)
    ap.add_argument("--coarse-steps", type=int, default=10000)
    ap.add_argument("--checkpoints", type=int, default=10)
    ap.add_argument("--snapshots", type=int, default=4)
    ap.add_argument("--train-steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=8)

    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--test-realizations", type=int, default=3)
    ap.add_argument("--fine-storage", default="f32")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    cfg = HitConfig(fine=a.fine, factor=a.factor, nu_fine=a.nu, coarse_steps=a.coarse_steps,
                    checkpoints=a.checkpoints, train_snapshots=a.snapshots, train_steps=a.train_steps,
                    closure_every=a.every, seed=a.seed, test_realizations=a.test_realizations,

                    fine_storage=zl.STORAGE_NAMES[a.fine_storage])
    res = run(cfg, log=lambda m: print(m, flush=True))
    out = {"config": res.config, "times": res.times, "errors": res.errors, "mlups": res.mlups,
           "training": res.training, "spectra": res.spectra}
    text = json.dumps(out)
    if a.out:
        with open(a.out, "w") as fh:
            fh.write(text)
    print(json.dumps({k: out[k] for k in ("errors", "mlups")}), flush=True)


if __name__ == "__main__":
    main()
