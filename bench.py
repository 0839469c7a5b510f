"""Benchmark: D3Q19 MRT Taylor-Green vortex on a periodic 256^3 lattice, one LBM time step per step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--storage f32|f16|bf16|f64] [--impl ours|reference]

Prints one JSON line (rank 0).  ``value`` is whole-job MLUPS over all ranks with the
populations resident in HBM; ``e2e`` is the same job through the C ABI with host buffers:
upload of the initial populations from pinned memory, K steps, read-back of density and
velocity, all inside the timed region.  The lattice (256^3 nodes, 2.55 GB of FP32
populations) is far larger than L2, so no flush is needed between steps.

Multi-GPU runs shard one lattice of 256 x 256 x 256N nodes into N slabs of 256^3 along z, one per
rank (weak scaling), with the two-stage halo exchange of the AA pattern over NCCL point-to-point
after every step (zllbm_b200.shard); ``--shard`` runs the same path at N = 1 as a one-rank periodic
ring, ``--replicas`` gives every rank its own lattice instead (no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "D3Q19 MLUPS & HBM-roofline %; learned vs Smagorinsky LES error at same GPU"
CELLS = 256          # unique nodes per axis (periodic; the reference stores 257 planes)
COLLISION = "mrt"
U0 = 0.05
TAU = 0.55
NU = (TAU - 0.5) / 3.0
STORAGE_BYTES = {"f64": 8, "f32": 4, "f16": 2, "bf16": 2}
FALLBACK_HBM_GBS = 6650.0


# ---------------------------------------------------------------- helpers
def tgv_nodes(cells: int, lo=(1, 1, 1), hi=None):
    """Morton codes of the reference's stored nodes (indices lo..hi per axis, by default 1..cells+1)
    and TGV feq populations (period `cells` on every axis), x fastest."""
    import zllbm_b200 as zl
    hi = hi or (cells + 1,) * 3
    codes = zl.box_codes(3, lo, hi)
    ax = [2.0 * np.pi * ((np.arange(lo[a], hi[a] + 1) - 1) % cells) / cells for a in range(3)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    x, y, z = x.ravel(), y.ravel(), z.ravel()
    ux = U0 * np.sin(x) * np.cos(y) * np.cos(z)
    uy = -U0 * np.cos(x) * np.sin(y) * np.cos(z)
    p = U0 * U0 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
    rho = 1.0 + 3.0 * p
    del x, y, z
    c = np.array([(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (1, 1, 0),
                  (-1, 1, 0), (1, -1, 0), (-1, -1, 0), (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1), (0, 1, 1),
                  (0, -1, 1), (0, 1, -1), (0, -1, -1)], dtype=np.float64)
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
    f = np.empty((codes.size, 19))
    usq = ux * ux + uy * uy
    for q in range(19):
        cu = ux * c[q, 0] + uy * c[q, 1]
        f[:, q] = w[q] * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq)
    return codes, f


def solver_config(storage: int, device: int):
    import zllbm_b200 as zl
    n = CELLS + 1
    return zl.SolverConfig(lattice=zl.D3Q19, collision=zl.MRT if COLLISION == "mrt" else zl.SRT,
                           storage=storage, viscosity=NU, rho0=1.0,
                           bc_kind=(zl.BC_PERIODIC,) * 6, domain_min=(1, 1, 1), domain_max=(n, n, n), device=device)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def committed_traffic(storage: str):
    """DRAM bytes per launch of the step kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            return json.load(fh).get(storage)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        exe = shutil.which("nvidia-smi")
        if exe:
            self.proc = subprocess.Popen([exe, f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- distributed plumbing
def dist_init(gpus: int):
    if gpus <= 1 or "RANK" not in os.environ:
        return 0, 1, int(os.environ.get("LOCAL_RANK", 0)), None
    import datetime

    import torch
    import torch.distributed as dist
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return dist.get_rank(), dist.get_world_size(), local, dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, value: float) -> float:
    """The slowest rank's time: every rank gets the maximum (NCCL reduces a device tensor, gloo a
    host one)."""
    if dist is None:
        return value
    import torch
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, value: float) -> float:
    if dist is None:
        return value
    import torch
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def whole_job_mlups(world: int, nodes_per_rank: int, steps: int, seconds: float) -> float:
    """Node updates of all replicas (each rank steps its own lattice: weak scaling) over the slowest
    rank's time."""
    return world * nodes_per_rank * steps / seconds / 1e6


# ---------------------------------------------------------------- CPU baselines
def reference_run(cells: int, steps: int, warmup: int, workdir: str):
    exe = os.path.join(ROOT, "oracle", "_ref", "zl_ref_run")
    args = [exe, "dims=3", f"n={cells},{cells},{cells}", f"steps={steps}", f"warmup={warmup}", "coll=mrt",
            f"nu={NU!r}", "init=tgv", f"u0={U0!r}", "timing=1"] + \
           [f"bc={f}:per" for f in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")]
    return subprocess.Popen(args, cwd=workdir, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)


def cpu_baseline_sample(processes: int = 1, cells: int = 48, steps: int = 30, warmup: int = 2):
    """Time the reference ZLLBM solver (oracle/_ref, built from its own sources) on a TGV
    subdomain of the same workload; `processes` independent single-rank runs model its MPI
    scaling across the host cores.  Falls back to the C restatement when the binary is absent."""
    import tempfile
    exe = os.path.join(ROOT, "oracle", "_ref", "zl_ref_run")
    nodes = (cells + 1) ** 3
    if os.path.exists(exe):
        with tempfile.TemporaryDirectory() as tmp:
            dirs = []
            for i in range(processes):
                d = os.path.join(tmp, str(i))
                os.makedirs(d)
                dirs.append(d)
            procs = [reference_run(cells, steps, warmup, d) for d in dirs]
            secs = []
            for p in procs:
                out, _ = p.communicate(timeout=1800)
                if p.returncode != 0:
                    raise RuntimeError("reference harness failed")
                secs.append(json.loads(out.strip().splitlines()[-1])["seconds"])
        wall = max(secs)
        mlups = processes * nodes * steps / wall / 1e6
        return {"value": mlups, "unit": "MLUPS", "cores": processes, "kind": "reference",
                "sample": f"reference ZLLBM TimeMarching, D3Q19 MRT TGV periodic {cells}^3 "
                          f"({nodes} stored nodes) x {steps} steps after {warmup} warm-up, "
                          f"{processes} single-rank process(es), max wall {wall:.2f} s"}
    from oracle.port import MRT, BC_PERIODIC, LevelConfig, Port, tgv_init
    port = Port()
    cfg = LevelConfig(dims=3, n=(cells + 1,) * 3, collision=MRT, nu=NU, bc_kind=(BC_PERIODIC,) * 6)
    f = tgv_init(cfg, U0, port).reshape(-1, 19)
    fc = f.copy()
    port.run(cfg, f, fc, warmup)
    t0 = time.perf_counter()
    port.run(cfg, f, fc, steps)
    wall = time.perf_counter() - t0
    return {"value": nodes * steps / wall / 1e6, "unit": "MLUPS", "cores": 1, "kind": "port",
            "sample": f"C restatement of the reference step, TGV {cells}^3 x {steps} steps, {wall:.2f} s"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return 0
    procs = max(1, min(os.cpu_count() or 1, 64))
    # bound the sample: about a minute of CPU work per process for K timed steps
    budget_lups = 60.0 * 0.8e6
    cells = int(max(16, min(64, round((budget_lups / max(args.steps, 1)) ** (1 / 3)) - 1)))
    cb = cpu_baseline_sample(processes=procs, cells=cells, steps=args.steps, warmup=args.warmup)
    out = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "MLUPS", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": "D3Q19 MRT Taylor-Green vortex, periodic, u0=0.05, tau=0.55 (sampled subdomain "
                                  f"{cells}^3 per process on the host cores)", "parallelism": f"{procs} processes"},
           "cpu_baseline": cb,
           "e2e": {"value": cb["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


# ---------------------------------------------------------------- GPU arm
def time_steps(ctx, steps: int, graph: bool = False):
    """Device time of `steps` time steps on the context's stream (CUDA events): zl_step_level
    per step, or zl_advance replaying the captured two-step graph."""
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream())
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    ctx.synchronize()
    start.record(stream)
    if graph:
        ctx.advance(steps)
    else:
        for _ in range(steps):
            ctx.step_level(0)
    end.record(stream)
    end.synchronize()
    return start.elapsed_time(end)


def closure_block():
    """The metric's second half: learned closure vs Smagorinsky on decaying HIT, measured on this
    GPU in this run on a reduced case (fine 256^3 -> coarse 64^3); the cost is measured on a 256^3
    coarse grid, the full case's."""
    from zllbm_b200.hit import HitConfig, run
    cfg = HitConfig(fine=256, factor=4, coarse_steps=2000, checkpoints=8, train_snapshots=4, train_steps=2000,
                    closure_every=16)
    t0 = time.perf_counter()
    res = run(cfg, log=lambda m: None)
    e = res.errors
    cost = res.mlups["cost"]
    return {
        "workload": "decaying HIT (seeded random-phase modes, k0=4, u_rms=0.04): fine D3Q19 SRT 256^3 box-filtered "
                    "by 4 to 64^3, 2000 coarse steps; trained and calibrated on one realization, scored on three "
                    "others (mean, spread)",
        "error": "RMS over shells and 8 checkpoints of log(E_LES / E_filtered_fine), lower is better",
        "test_realizations": len(e["smagorinsky"]["per_realization"]),
        "smagorinsky_cs0.1": e["smagorinsky"]["error"],
        "smagorinsky_calibrated": e["smagorinsky_calibrated"]["error"],
        "learned_calibrated": e["learned_calibrated"]["error"],
        "learned_calibrated_every16": e["learned_calibrated_every16"]["error"],
        "error_std": {k: e[k]["error_std"] for k in ("smagorinsky", "smagorinsky_calibrated", "learned_calibrated",
                                                       "learned_calibrated_every16")},
        "learned_minus_smagorinsky_calibrated": e["learned_minus_smagorinsky_calibrated"],
        "alpha": res.training["alpha"], "cs_calibrated": res.training["calibration"]["cs_best"],
        "held_out_mse": {"network": res.training["val_loss"], "smagorinsky_y1": res.training["val_loss_smagorinsky_y1"],
                         "best_constant": res.training["val_loss_best_constant"]},
        "mlups_256": {k: cost[k] for k in ("smagorinsky", "learned", "learned_every8", "learned_every16")},
        "cost_fraction_every16": cost["learned_every16_cost_fraction"],
        "cost_fraction_every_step": cost["learned_cost_fraction"],
        "seconds": time.perf_counter() - t0,
    }


def kernel_name(block, storage: str) -> str:
    """The step kernel the (autotuned) block shape selects."""
    import zllbm_b200 as zl
    if block and block[0] == zl.BLOCK_ROW:
        return f"aa_row_kernel<{storage}, {COLLISION.upper()}> (one warp per x-row)"
    if block and block[0] < 0:
        return f"aa_pair_kernel<{storage}, {COLLISION.upper()}> (two nodes per thread)"
    return f"aa_step_kernel<D3Q19, {storage}, {COLLISION.upper()}>"


def multilevel_block(steps: int, warmup: int, peak: float):
    """The multi-level configurations on the reference-built grids (packed under
    zllbm_b200/topologies/): the cube flow (D3Q19 SRT + Smagorinsky + immersed-boundary cube,
    levels 0..2) and the cylinder flow (D2Q9 MRT + immersed-boundary cylinder, levels 0..3), FP32,
    per-level streams replayed from a CUDA graph.  MLUPS count every node update of every level
    (nodes x 2^level per coarse step); the HBM figure is those updates' algorithmic bytes
    (2 Q sizeof(float) each) over the event time."""
    from zllbm_b200 import cube_flow, cylinder_flow
    out = {}
    for name, mod, q, k in (("cube_flow", cube_flow, 19, steps), ("cylinder_flow", cylinder_flow, 9, 4 * steps)):
        res = mod.run(mod.DEFAULT_TOPOLOGY, steps=k, warmup=warmup, log=lambda m: None)
        gbs = res["mlups"] * 1e6 * 2 * q * 4 / 1e9
        out[name] = {"workload": res["workload"], "mlups": res["mlups"], "ms_per_coarse_step": res["ms_per_coarse_step"],
                     "coarse_steps": k, "nodes_per_level": res["nodes_per_level"],
                     "hbm_gbs_algorithmic": gbs, "frac": gbs / peak, "finite": res["finite"]}
    return out


def run_ours(args):
    import torch

    import zllbm_b200 as zl
    rank, world, local, dist = dist_init(args.gpus)
    torch.cuda.set_device(local)
    if args.shard or (world > 1 and not args.replicas):
        return run_sharded(args, rank, world, local, dist)
    storage = zl.STORAGE_NAMES[args.storage]
    elem = STORAGE_BYTES[args.storage]
    codes, f0 = tgv_nodes(CELLS)
    nodes = CELLS ** 3
    alg_bytes = nodes * 2 * 19 * elem  # read + write every population once per update

    ctx = zl.Context(solver_config(storage, local))
    ctx.set_level_nodes(0, codes)
    ctx.set_populations(0, codes, f0)
    block = ctx.autotune(0) if args.tune else None
    if args.tune:
        ctx.set_populations(0, codes, f0)
    ctx.set_graph(args.graph)
    # the graph is captured by the first zl_advance of two or more steps, inside the warm-up
    if args.graph:
        ctx.advance(args.warmup)
    else:
        for _ in range(args.warmup):
            ctx.step_level(0)
    ctx.synchronize()
    mass_before = ctx.conservation(0)[0]  # outside the timed region

    barrier(dist)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ms = time_steps(ctx, args.steps, args.graph)
    torch.cuda.synchronize()
    barrier(dist)
    ms = max_over_ranks(dist, ms)
    mass = ctx.conservation(0)[0]

    ms_per_step = ms / args.steps
    value = whole_job_mlups(world, nodes, args.steps, ms / 1e3)
    peak, peak_kind = measured_peak()
    achieved = alg_bytes / (ms_per_step / 1e3) / 1e9
    traffic = committed_traffic(args.storage)

    # other storage precisions of the same workload, kernel time only (reported alongside)
    variants = {}
    if args.variants and rank == 0:
        # 16-bit storages with the default stochastic rounding and ("rn") round to nearest
        for name in ("f16", "bf16", "f32", "f16rn", "bf16rn"):
            if name == args.storage:
                continue
            rn = name.endswith("rn")
            base = name[:-2] if rn else name
            vcfg = solver_config(zl.STORAGE_NAMES[base], local)
            vcfg.storage_rounding = zl.ROUND_NEAREST if rn else zl.ROUND_STOCHASTIC
            with zl.Context(vcfg) as c2:
                c2.set_level_nodes(0, codes)
                c2.set_populations(0, codes, f0)
                vblock = c2.autotune(0) if args.tune else None
                if args.tune:
                    c2.set_populations(0, codes, f0)
                c2.set_graph(args.graph)
                c2.advance(args.warmup)
                vms = time_steps(c2, args.steps, args.graph)
                b = nodes * 2 * 19 * STORAGE_BYTES[base]
                variants[name] = {"mlups": nodes * args.steps / (vms / 1e3) / 1e6,
                                  "ms_per_step": vms / args.steps,
                                  "hbm_gbs": b / (vms / args.steps / 1e3) / 1e9,
                                  "frac": b / (vms / args.steps / 1e3) / 1e9 / peak,
                                  "block": vblock, "kernel": kernel_name(vblock, name),
                                  "rounding": "nearest" if rn else ("stochastic" if base in ("f16", "bf16") else None)}
    # end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        f_h = torch.from_numpy(f0).pin_memory()
        rho_h = torch.empty(codes.size, dtype=torch.float64).pin_memory()
        u_h = torch.empty((codes.size, 3), dtype=torch.float64).pin_memory()
        lib = ctx.lib
        import ctypes
        dp = ctypes.POINTER(ctypes.c_double)
        # the level's node list was handed over once (zl_set_level_nodes); exchanges without codes
        # use it in that order, so only populations and fields cross PCIe
        barrier(dist)
        ctx.synchronize()
        t0 = time.perf_counter()
        ctx._check(lib.zl_set_populations(ctx.handle, 0, None, ctypes.cast(f_h.data_ptr(), dp), codes.size))
        ctx._check(lib.zl_advance(ctx.handle, args.steps))
        ctx._check(lib.zl_get_macros(ctx.handle, 0, None, ctypes.cast(rho_h.data_ptr(), dp),
                                     ctypes.cast(u_h.data_ptr(), dp), codes.size))
        ctx.synchronize()
        t_e2e = max_over_ranks(dist, time.perf_counter() - t0)
        h2d = f0.nbytes
        d2h = rho_h.numel() * 8 + u_h.numel() * 8
        e2e = {"value": whole_job_mlups(world, nodes, args.steps, t_e2e), "unit": "MLUPS",
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "seconds": t_e2e,
               "includes": "H2D of the initial populations (pinned; node codes handed over once at set-up), "
                           "K steps, D2H of rho and u"}
    ctx.close()

    multilevel = multilevel_block(max(16, args.steps), args.warmup, peak) if rank == 0 and args.multilevel else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(processes=1)
    closure = closure_block() if rank == 0 and args.closure else None
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.storage, "data": "synthetic",
            "config": {"workload": f"D3Q19 {COLLISION.upper()} Taylor-Green vortex, periodic {CELLS}^3 "
                                   f"(reference stores {CELLS + 1}^3), u0={U0}, tau={TAU}, "
                                   f"{args.storage} population storage, "
                                   + ("FP64 collision" if args.storage == "f64" else "FP32 collision"),
                       "block": block, "cuda_graph": args.graph,
                       "nodes_per_gpu": nodes, "storage": args.storage, "collision": COLLISION.upper(),
                       "l2": f"inputs larger than L2 ({alg_bytes / 2 / 1e9:.2f} GB of populations)",
                       "parallelism": f"{world} independent replica(s)" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_kind": peak_kind, "algorithmic_bytes_per_launch": alg_bytes,
                         "kernel": kernel_name(block, args.storage)},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": args.steps,
            "clocks": clocks.summary(),
            "mass_after": mass,
            "mass_drift": (mass - mass_before) / mass_before,
        }
        if variants:
            out["storage_variants"] = variants
        if multilevel:
            out["multilevel"] = multilevel
        if closure:
            out["closure"] = closure
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_sharded(args, rank: int, world: int, local: int, dist):
    """One lattice of CELLS x CELLS x (CELLS world) nodes, periodic, split into `world` slabs of
    CELLS planes along z (zllbm_b200.shard): each rank steps its slab and swaps halo planes with its
    two neighbours after every step (NCCL point-to-point; at world 1 the ring routes the buffers to
    itself).  The Taylor-Green field repeats with period CELLS along z, so every slab starts as the
    single-GPU workload."""
    import ctypes

    import torch

    import zllbm_b200 as zl
    from zllbm_b200.shard import DeviceSlab, LocalRing, Ring, SlabSchedule, torch_exchange
    storage = zl.STORAGE_NAMES[args.storage]
    elem = STORAGE_BYTES[args.storage]
    gcfg = solver_config(storage, local)
    gcfg.domain_max = (CELLS + 1, CELLS + 1, CELLS * world + 1)
    ring = Ring(rank, world, True)
    lo, hi = rank * CELLS, (rank + 1) * CELLS
    slab = DeviceSlab(gcfg, lo, hi, ring)
    codes, f0 = tgv_nodes(CELLS, (1, 1, 1 + lo), (CELLS + 1, CELLS + 1, hi))
    if not np.array_equal(codes, slab.codes):
        raise RuntimeError("slab node order")
    nodes = CELLS ** 3
    alg_bytes = nodes * 2 * 19 * elem
    ctx = slab.ctx
    ctx.set_populations(0, None, f0)
    block = ctx.autotune(0) if args.tune else None
    if args.tune:
        ctx.set_populations(0, None, f0)
    # the overlapped schedule: interior planes step while the previous step's halo is in flight
    sched = LocalRing([slab], True, slab.faces, overlap=True) if world == 1 else \
        SlabSchedule(slab, ring, slab.faces, torch_exchange(dist), overlap=True)
    barrier(dist)  # every rank's communicator is up before the first point-to-point exchange
    for _ in range(args.warmup):
        sched.step()
    sched.flush()
    mass_before = sum_over_ranks(dist, ctx.conservation(0)[0])
    stream = torch.cuda.current_stream()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            sched.step()
        sched.flush()
        end.record(stream)
        end.synchronize()
    torch.cuda.synchronize()
    barrier(dist)
    ms = max_over_ranks(dist, start.elapsed_time(end))
    mass = sum_over_ranks(dist, ctx.conservation(0)[0])
    ms_per_step = ms / args.steps
    value = whole_job_mlups(world, nodes, args.steps, ms / 1e3)
    peak, peak_kind = measured_peak()
    achieved = alg_bytes / (ms_per_step / 1e3) / 1e9
    halo_bytes = sum(slab.nbytes.values())

    e2e = None
    if not args.no_e2e:
        f_h = torch.from_numpy(f0).pin_memory()
        rho_h = torch.empty(codes.size, dtype=torch.float64).pin_memory()
        u_h = torch.empty((codes.size, 3), dtype=torch.float64).pin_memory()
        dp = ctypes.POINTER(ctypes.c_double)
        lib = ctx.lib
        barrier(dist)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx._check(lib.zl_set_populations(ctx.handle, 0, None, ctypes.cast(f_h.data_ptr(), dp), codes.size))
        for _ in range(args.steps):
            sched.step()
        sched.flush()
        ctx._check(lib.zl_get_macros(ctx.handle, 0, None, ctypes.cast(rho_h.data_ptr(), dp),
                                     ctypes.cast(u_h.data_ptr(), dp), codes.size))
        torch.cuda.synchronize()
        t_e2e = max_over_ranks(dist, time.perf_counter() - t0)
        e2e = {"value": whole_job_mlups(world, nodes, args.steps, t_e2e), "unit": "MLUPS",
               "h2d_bytes_per_step": f0.nbytes / args.steps,
               "d2h_bytes_per_step": (rho_h.numel() + u_h.numel()) * 8 / args.steps, "seconds": t_e2e,
               "includes": "per rank: H2D of its slab's initial populations (pinned), K steps with their halo "
                           "exchanges, D2H of rho and u"}
    slab.close()
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.storage, "data": "synthetic",
            "config": {"workload": f"D3Q19 {COLLISION.upper()} Taylor-Green vortex, periodic {CELLS} x {CELLS} x "
                                   f"{CELLS * world} (z period {CELLS}), u0={U0}, tau={TAU}, "
                                   f"{args.storage} population storage",
                       "block": block, "cuda_graph": False, "nodes_per_gpu": nodes, "storage": args.storage,
                       "collision": COLLISION.upper(),
                       "l2": f"inputs larger than L2 ({alg_bytes / 2 / 1e9:.2f} GB of populations per GPU)",
                       "parallelism": f"slab sharding along z over {world} GPU(s), halo exchange after every step "
                                      + ("(NCCL point-to-point)" if world > 1 else "(one-rank ring, device copies)")
                                      + ", interior planes stepped while the halo is in flight",
                       "halo_bytes_per_exchange": halo_bytes},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": committed_traffic(args.storage), "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes, "kernel": kernel_name(block, args.storage),
                         "note": "step time includes the halo packs, exchanges and unpacks"},
            "cpu_baseline": None,
            "e2e": e2e,
            # per step: the step kernel in three plane ranges, a pack per face and an unpack per face
            "gpu_launches": args.steps * 7,
            "clocks": clocks.summary(),
            "mass_after": mass,
            "mass_drift": (mass - mass_before) / mass_before,
        }
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--storage", default="f32", choices=sorted(STORAGE_BYTES))
    ap.add_argument("--cells", type=int, default=256, help="lattice edge (256 is the benchmark workload)")
    ap.add_argument("--collision", default="mrt", choices=["mrt", "srt"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--variants", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--closure", type=int, default=1, help="learned-closure vs Smagorinsky block (HIT, ~40 s)")
    ap.add_argument("--tune", type=int, default=1, help="autotune the step kernel's block shape")
    ap.add_argument("--graph", type=int, default=1, help="replay steps as a captured CUDA graph")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shard", action="store_true", help="slab-sharded path at any N (N = 1: one-rank ring)")
    ap.add_argument("--replicas", action="store_true", help="N > 1: independent lattices instead of slabs")
    ap.add_argument("--multilevel", type=int, default=1,
                    help="multi-level cube-flow and cylinder-flow block (reference-built grids)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    globals()["CELLS"] = args.cells
    globals()["COLLISION"] = args.collision
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
