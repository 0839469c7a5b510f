"""Storage-precision study on the D3Q19 MRT Taylor-Green vortex (periodic box, u0 = 0.05,
tau = 0.55): the same run in FP64, FP32, FP16-deviation and BF16-deviation storage, with the
velocity's relative L2 error against the FP64 run and the kinetic-energy decay at checkpoints.

    python -m zllbm_b200.tgv_accuracy [--cells 256] [--steps 5000] [--checkpoints 5] [--out file.json]
                                      [--storages f32,f16,f16rn,bf16,bf16rn]

FP64 storage is the device path that is bit-exact to the reference's own solver, so it is the
FP64 oracle of the comparison.  Every run starts from feq(rho, u) of the analytic TGV fields
(pressure from the TGV formula, rho = 1 + 3 p).  Kinetic energy is also compared with the
linear viscous decay exp(-2 nu |k|^2 t), |k|^2 = 3 (2 pi / N)^2 (the u0 = 0.05 vortex is nearly
linear at these Reynolds numbers).  Each error is also split into an amplitude part (the
projection on the FP64 field, a = <u, u64> / <u64, u64>: a - 1 is a decay-rate bias) and the part
orthogonal to it (|u - a u64| / |u64|: noise and shape errors).  FP16 / BF16 store with the
library's default stochastic rounding; a name ending in "rn" (f16rn, bf16rn) rounds to nearest.  The 16-bit runs take the
benchmark's kernel where it applies (one warp per x-row for 128- and 256-node rows).
"""
from __future__ import annotations

import argparse
import json
import math
import time

import zllbm_b200 as zl

U0 = 0.05
TAU = 0.55


def tgv_fields(n: int):
    import torch
    ax = 2.0 * math.pi * torch.arange(n, device="cuda", dtype=torch.float64) / n
    z, y, x = torch.meshgrid(ax, ax, ax, indexing="ij")
    u = torch.stack([U0 * torch.sin(x) * torch.cos(y) * torch.cos(z),
                     -U0 * torch.cos(x) * torch.sin(y) * torch.cos(z),
                     torch.zeros_like(x)], dim=-1).reshape(-1, 3).float().contiguous()
    p = U0 * U0 / 16.0 * (torch.cos(2 * x) + torch.cos(2 * y)) * (torch.cos(2 * z) + 2.0)
    rho = (1.0 + 3.0 * p).reshape(-1).float().contiguous()
    return rho, u


def run_storage(storage: str, n: int, steps: int, checkpoints: int, log=print):
    """Velocity fields (FP32, box order) at the checkpoints and the MLUPS of the run."""
    import torch
    from zllbm_b200.hit import box_context
    every = steps // checkpoints
    out = []
    rn = storage.endswith("rn")
    base = storage[:-2] if rn else storage
    with torch.cuda.stream(torch.cuda.Stream()):
        ctx = box_context(n, TAU, storage=zl.STORAGE_NAMES[base], collision=zl.MRT,
                          rounding=zl.ROUND_NEAREST if rn else zl.ROUND_STOCHASTIC)
        if zl.STORAGE_NAMES[base] in (zl.STORAGE_F16, zl.STORAGE_BF16) and n in (128, 256):
            ctx.set_block(0, zl.BLOCK_ROW, 1)
        rho, u = tgv_fields(n)
        ctx.set_equilibrium_dense(0, rho.data_ptr(), u.data_ptr())
        ctx.synchronize()
        t0 = time.perf_counter()
        done = 0
        for c in range(checkpoints):
            for _ in range(every):
                ctx.step_level(0)
            done += every
            ctx.get_macros_dense(0, rho.data_ptr(), u.data_ptr())
            ctx.synchronize()
            out.append((done, u.clone()))
        seconds = time.perf_counter() - t0
        ctx.close()
    mlups = n ** 3 * done / seconds / 1e6
    log(f"{storage}: {done} steps in {seconds:.2f} s (with read-backs): {mlups:.0f} MLUPS")
    return out, mlups


def run(n: int = 256, steps: int = 5000, checkpoints: int = 5, log=print,
        storages: tuple = ("f32", "f16", "f16rn", "bf16", "bf16rn")) -> dict:
    import torch
    nu = (TAU - 0.5) / 3.0
    k2 = 3.0 * (2.0 * math.pi / n) ** 2
    ref, mlups64 = run_storage("f64", n, steps, checkpoints, log)
    e0 = U0 * U0 / 8.0  # <u^2 + v^2> / 2 of the initial field: u0^2 (1/8 + 1/8) / 2
    result = {"workload": f"D3Q19 MRT TGV periodic {n}^3, u0={U0}, tau={TAU}, {steps} steps, "
                          "initial feq of the analytic fields",
              "steps_at": [s for s, _ in ref], "storages": {}}
    ke_ref = [float(0.5 * (u.double() ** 2).sum(1).mean()) for _, u in ref]
    result["kinetic_energy_f64"] = ke_ref
    result["kinetic_energy_linear_decay"] = [e0 * math.exp(-2.0 * nu * k2 * s) for s, _ in ref]
    result["storages"]["f64"] = {"mlups_with_readback": mlups64}
    for storage in storages:
        fields, mlups = run_storage(storage, n, steps, checkpoints, log)
        errs, kes, amps, perps = [], [], [], []
        for (s, u), (_, u64) in zip(fields, ref):
            ud, rd = u.double(), u64.double()
            nr = rd.norm()
            diff = (ud - rd).norm() / nr
            a = float((ud * rd).sum() / (nr * nr))
            errs.append(float(diff))
            amps.append(a - 1.0)
            perps.append(float((ud - a * rd).norm() / nr))
            kes.append(float(0.5 * (ud ** 2).sum(1).mean()))
        result["storages"][storage] = {"velocity_rel_l2_vs_f64": errs, "amplitude_minus_1": amps,
                                       "orthogonal_rel_l2": perps, "kinetic_energy": kes,
                                       "kinetic_energy_rel_diff_vs_f64": [k / r - 1.0 for k, r in zip(kes, ke_ref)],
                                       "mlups_with_readback": mlups}
        log(f"{storage}: velocity rel L2 vs FP64 at checkpoints {['%.2e' % e for e in errs]}")
        del fields
        torch.cuda.empty_cache()
    return result


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--cells", type=int, default=256)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--checkpoints", type=int, default=5)
    ap.add_argument("--out", default=None)
    ap.add_argument("--storages", default="f32,f16,f16rn,bf16,bf16rn")
    a = ap.parse_args(argv)
    res = run(a.cells, a.steps, a.checkpoints, storages=tuple(a.storages.split(",")))
    text = json.dumps(res, indent=1)
    if a.out:
        with open(a.out, "w") as fh:
            fh.write(text)
    print(text)


if __name__ == "__main__":
    main()
