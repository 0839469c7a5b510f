"""Small single-kernel workloads for profiling (one launch type each, few launches).

    python -m zllbm_b200.kernel_cases step --storage f16 --cells 192 [--collision mrt] [--block 128|-64|row]
        [--block-y 1]
    python -m zllbm_b200.kernel_cases learned --cells 128
    python -m zllbm_b200.kernel_cases train [--samples 151552]

``step``: a periodic Taylor-Green box level, 6 plain steps (no CUDA graph) of the fused
collide-stream kernel.  ``learned``: a periodic HIT box level with the learned closure evaluated
in the step (4 steps of learned_step_kernel).  ``train``: 3 Adam steps of the device trainer on
random features.  Each runs 2 untimed warm-up launches first and prints its throughput, timed with
CUDA events on the library's stream.
"""
from __future__ import annotations

import argparse
import math

import zllbm_b200 as zl


def _events(stream, fn, reps: int, warmup: int = 2) -> float:
    import torch
    s = torch.cuda.ExternalStream(stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a.record(s)
    for _ in range(reps):
        fn()
    b.record(s)
    b.synchronize()
    return a.elapsed_time(b)


def step_case(storage: str, cells: int, collision: str, block: int, steps: int = 6, block_y: int = 1) -> float:
    import torch
    from zllbm_b200.hit import box_context
    u0 = 0.05
    with torch.cuda.stream(torch.cuda.Stream()):
        ctx = box_context(cells, 0.55, storage=zl.STORAGE_NAMES[storage],
                          collision=zl.MRT if collision == "mrt" else zl.SRT)
        ax = 2.0 * math.pi * torch.arange(cells, device="cuda", dtype=torch.float64) / cells
        z, y, x = torch.meshgrid(ax, ax, ax, indexing="ij")
        u = torch.stack([u0 * torch.sin(x) * torch.cos(y) * torch.cos(z),
                         -u0 * torch.cos(x) * torch.sin(y) * torch.cos(z),
                         torch.zeros_like(x)], dim=-1).reshape(-1, 3).float().contiguous()
        p = u0 * u0 / 16.0 * (torch.cos(2 * x) + torch.cos(2 * y)) * (torch.cos(2 * z) + 2.0)
        rho = (1.0 + 3.0 * p).reshape(-1).float().contiguous()
        del x, y, z, p
        ctx.set_equilibrium_dense(0, rho.data_ptr(), u.data_ptr())
        if block:
            ctx.set_block(0, block, block_y)
        ms = _events(ctx.stream(), lambda: ctx.step_level(0), steps)
        ctx.close()
    mlups = cells ** 3 * steps / (ms * 1e-3) / 1e6
    shape = "default" if not block else ("row" if block == zl.BLOCK_ROW else str(block))
    print(f"step {storage} {collision} {cells}^3 block {shape} x {block_y}: {mlups:.0f} MLUPS", flush=True)
    return mlups


def learned_case(cells: int, steps: int = 4) -> float:
    import torch
    from zllbm_b200.hit import box_context, hit_velocity, initial_net
    with torch.cuda.stream(torch.cuda.Stream()):
        u = hit_velocity(cells)
        rho = torch.ones(cells ** 3, device="cuda")
        ctx = box_context(cells, 0.5015, les=zl.LES_LEARNED, cs=0.1)
        ctx.set_closure(initial_net(3))
        ctx.set_equilibrium_dense(0, rho.data_ptr(), u.data_ptr())
        ms = _events(ctx.stream(), lambda: ctx.step_level(0), steps)
        ctx.close()
    mlups = cells ** 3 * steps / (ms * 1e-3) / 1e6
    print(f"learned {cells}^3: {mlups:.0f} MLUPS", flush=True)
    return mlups


def train_case(samples: int, steps: int = 3) -> float:
    import torch
    from zllbm_b200.hit import initial_net
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    x = torch.randn(samples, zl.MLP_IN, device="cuda", generator=g)
    y = torch.rand(samples, device="cuda", generator=g)
    with zl.Trainer(initial_net(1)) as tr:
        tr.set_stream(torch.cuda.current_stream().cuda_stream)
        ms = _events(torch.cuda.current_stream().cuda_stream,
                     lambda: tr.step(x.data_ptr(), y.data_ptr(), samples, 1e-3), steps)
        loss = tr.loss()
    rate = samples * steps / (ms * 1e-3) / 1e6
    print(f"train {samples} samples x {steps} steps: {rate:.1f} M samples/s, last batch loss {loss:.4g}", flush=True)
    return rate


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("case", choices=["step", "learned", "train"])
    ap.add_argument("--storage", default="f32", choices=sorted(zl.STORAGE_NAMES))
    ap.add_argument("--collision", default="mrt", choices=["mrt", "srt"])
    ap.add_argument("--cells", type=int, default=192)
    ap.add_argument("--block", default="0",
                    help="block x of the step kernel (0: library default; negative: two nodes per thread; "
                         "row: one warp per x-row)")
    ap.add_argument("--block-y", type=int, default=1, help="block y (row kernel: rows per block)")
    ap.add_argument("--samples", type=int, default=128 * 148 * 8)
    a = ap.parse_args(argv)
    if a.case == "step":
        block = zl.BLOCK_ROW if a.block == "row" else int(a.block)
        step_case(a.storage, a.cells, a.collision, block, block_y=a.block_y)
    elif a.case == "learned":
        learned_case(a.cells)
    else:
        train_case(a.samples)


if __name__ == "__main__":
    main()
