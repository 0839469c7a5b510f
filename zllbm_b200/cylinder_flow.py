"""Multi-level flow past a cylinder: D2Q9 MRT on a coarse 1024 x 512 domain with three refinement
levels (factor 2 each, sub-cycled 1:2:4:8) around a cylinder of diameter 40 finest cells (5 coarse
cells), inflow 0.04 (non-equilibrium extrapolation), convective outflow, bounce-back side walls,
Re = 200 on the diameter, FP32 storage; the cylinder is 400 immersed-boundary vertices on the
finest level (direct forcing with the reference's four-point delta kernel).  The levels' steps,
passes and transfers run on per-level streams, replayed from a CUDA graph; drag and lift are the FP64 sums of the vertex
forces.

    python -m zllbm_b200.cylinder_flow [--topology cylinder_topology.npz] [--steps 400] [--warmup 8]

The node sets and interface layers come from the host's grid builder: the reference's own
(``oracle/make_body_topology.py --n 1024,512 --levels 3 --circle 256,256,2.5 --ext 8 --inner 8``);
the default, ``zllbm_b200/topologies/cylinder_1024x512_l3.npz``, is that grid in the packed form
of ``zllbm_b200.topology_pack``.  Throughput counts
every node update the reference performs: the sum over levels of nodes x 2^level per coarse step.
"""
from __future__ import annotations

import argparse
import json
import os
import math
import time

import numpy as np

import zllbm_b200 as zl
from zllbm_b200.topology_pack import load_topology

DEFAULT_TOPOLOGY = os.path.join(os.path.dirname(os.path.abspath(__file__)), "topologies", "cylinder_1024x512_l3.npz")

U_IN = 0.04
RE = 200.0
VERTICES = 400


def build(topology: str, storage: int = zl.STORAGE_F32):
    z = load_topology(topology)
    meta = json.loads(str(z["meta"]))
    levels = meta["levels"]
    n = meta["n"]
    cx, cy, r = (float(v) for v in meta["circle"].split(","))
    nu = U_IN * 2.0 * r / RE
    walls = zl.BC_BOUNCE_BACK
    cfg = zl.SolverConfig(lattice=zl.D2Q9, collision=zl.MRT, storage=storage, max_level=levels, viscosity=nu,
                          bc_kind=(zl.BC_NONEQ_EXTRAPOLATION, zl.BC_CONVECTIVE_OUTFLOW, walls, walls, 0, 0),
                          bc_velocity=((U_IN, 0.0, 0.0), (U_IN, 0.0, 0.0)) + ((0.0, 0.0, 0.0),) * 4,
                          domain_min=(1, 1, 0), domain_max=(n[0] + 1, n[1] + 1, 0),
                          init_velocity=(U_IN, 0.0, 0.0), forcing=1)
    ctx = zl.Context(cfg)
    nodes = []
    for lv in range(levels + 1):
        ctx.set_level_nodes(lv, z[f"codes{lv}"])
        nodes.append(int(z[f"codes{lv}"].size))
    for lv in range(1, levels + 1):
        excluded = z[f"codes{lv - 1}"][(z[f"flags{lv - 1}"] & 4) != 0]
        ctx.set_level_interface(lv, z[f"c2f_fine{lv}"], z[f"f2c_coarse{lv - 1}"], excluded)
    t = 2.0 * math.pi * np.arange(VERTICES) / VERTICES
    xyz = np.stack([cx + r * np.cos(t), cy + r * np.sin(t), np.zeros(VERTICES)], axis=1)
    arc = np.full(VERTICES, 2.0 * math.pi * r / VERTICES)
    ctx.ib_set_vertices(levels, xyz, np.zeros_like(xyz), arc)
    return ctx, meta, nodes


def run(topology: str, steps: int = 400, warmup: int = 8, graph: bool = True, batching: bool = True, streams: bool = True,
        log=print) -> dict:
    import torch
    ctx, meta, nodes = build(topology)
    levels = meta["levels"]
    lups_per_step = sum(n * (1 << lv) for lv, n in enumerate(nodes))
    ctx.set_batching(batching)
    ctx.set_level_streams(streams)
    ctx.set_graph(graph)
    ctx.advance(warmup)
    ctx.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    ctx.advance(steps)
    b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b)
    force = ctx.ib_get_forces(levels)[1]
    ctx.close()
    diameter = 2.0 * float(meta["circle"].split(",")[2]) * (1 << levels)
    cycles = ":".join(str(1 << lv) for lv in range(levels + 1))
    res = {"workload": f"D2Q9 MRT flow past a cylinder (D = {diameter:g} finest cells, {VERTICES} immersed-boundary "
                       f"vertices), coarse {'x'.join(str(v) for v in meta['n'])}, {levels} refinement levels "
                       f"({cycles} sub-cycling), inflow {U_IN}, "
                       f"convective outflow, Re {RE:.0f}, FP32",
           "batched_level_steps": batching and not streams, "level_streams": streams, "cuda_graph": graph,
           "nodes_per_level": nodes, "lups_per_coarse_step": lups_per_step, "coarse_steps": steps,
           "ms_per_coarse_step": ms / steps, "mlups": lups_per_step * steps / (ms * 1e-3) / 1e6,
           "cylinder_force_total_fp64": [float(v) for v in force],
           "finite": bool(np.all(np.isfinite(force)))}
    log(json.dumps(res))
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--topology", default=DEFAULT_TOPOLOGY)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--graph", type=int, default=1)
    ap.add_argument("--batching", type=int, default=1)
    ap.add_argument("--streams", type=int, default=1, help="per-level streams (zl_set_level_streams)")
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    run(a.topology, a.steps, a.warmup, bool(a.graph), bool(a.batching), bool(a.streams))
    print(f"wall {time.perf_counter() - t0:.1f} s")


if __name__ == "__main__":
    main()
