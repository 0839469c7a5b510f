"""Multi-level flow past a cube: D3Q19 SRT + Smagorinsky (Cs = 0.1) on a coarse 256 x 128 x 128
domain with two refinement levels (factor 2 each, sub-cycled 1:2:4) around a cube of 16 coarse
cells, inflow 0.05 (non-equilibrium extrapolation), convective outflow, bounce-back side walls,
Re = 1000 on the cube edge, FP32 storage; the cube is an immersed boundary (direct forcing, its
surface vertices on the finest level).  The levels' steps, passes and transfers run on per-level
streams (the background step overlapping the finer levels' sub-steps), replayed from a CUDA graph.

    python -m zllbm_b200.cube_flow [--topology cube_topology.npz] [--steps 64] [--warmup 4]

The node sets and interface layers come from the host's grid builder: the reference's own
(``oracle/make_body_topology.py`` writes them from its AmrManager::SetupMesh).  The default,
``zllbm_b200/topologies/cube_256x128x128_l2.npz``, is that builder's grid for this case
(``--n 256,128,128 --levels 2 --cube 80,64,64,16 --ext 6 --inner 16``) in the packed form of
``zllbm_b200.topology_pack``.  Throughput counts
every node update the reference performs: the sum over levels of nodes x 2^level per coarse
step.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

import zllbm_b200 as zl
from zllbm_b200.topology_pack import load_topology

DEFAULT_TOPOLOGY = os.path.join(os.path.dirname(os.path.abspath(__file__)), "topologies", "cube_256x128x128_l2.npz")

U_IN = 0.05
RE = 1000.0


def cube_vertices(center, edge: float, h: float) -> tuple[np.ndarray, np.ndarray]:
    """Surface points of an axis-aligned cube on a grid of spacing h (shared edges once) and the
    area each represents."""
    m = int(round(edge / h))
    t = np.linspace(-edge / 2, edge / 2, m + 1)
    pts = set()
    for axis in range(3):
        for side in (-edge / 2, edge / 2):
            for a in t:
                for b in t:
                    p = [0.0, 0.0, 0.0]
                    p[axis] = side
                    p[(axis + 1) % 3] = a
                    p[(axis + 2) % 3] = b
                    pts.add(tuple(round(v / h) for v in p))
    xyz = np.array(sorted(pts), dtype=np.float64) * h + np.asarray(center, dtype=np.float64)
    area = np.full(len(xyz), 6.0 * edge * edge / len(xyz))
    return xyz, area


def build(topology: str, storage: int = zl.STORAGE_F32):
    z = load_topology(topology)
    meta = json.loads(str(z["meta"]))
    levels = meta["levels"]
    n = meta["n"]
    cx, cy, cz, edge = (float(v) for v in meta["cube"].split(","))
    nu = U_IN * edge / RE
    walls = zl.BC_BOUNCE_BACK
    cfg = zl.SolverConfig(lattice=zl.D3Q19, collision=zl.SRT, storage=storage, max_level=levels, viscosity=nu,
                          bc_kind=(zl.BC_NONEQ_EXTRAPOLATION, zl.BC_CONVECTIVE_OUTFLOW, walls, walls, walls, walls),
                          bc_velocity=((U_IN, 0.0, 0.0), (U_IN, 0.0, 0.0)) + ((0.0, 0.0, 0.0),) * 4,
                          domain_min=(1, 1, 1), domain_max=(n[0] + 1, n[1] + 1, n[2] + 1),
                          init_velocity=(U_IN, 0.0, 0.0), forcing=1, les=zl.LES_SMAGORINSKY, les_cs=0.1)
    ctx = zl.Context(cfg)
    nodes = []
    for lv in range(levels + 1):
        ctx.set_level_nodes(lv, z[f"codes{lv}"])
        nodes.append(int(z[f"codes{lv}"].size))
    for lv in range(1, levels + 1):
        excluded = z[f"codes{lv - 1}"][(z[f"flags{lv - 1}"] & 4) != 0]
        ctx.set_level_interface(lv, z[f"c2f_fine{lv}"], z[f"f2c_coarse{lv - 1}"], excluded)
    xyz, area = cube_vertices((cx, cy, cz), edge, 1.0 / (1 << levels))
    ctx.ib_set_vertices(levels, xyz, np.zeros_like(xyz), area)
    return ctx, meta, nodes, len(xyz)


def run(topology: str, steps: int = 64, warmup: int = 4, graph: bool = True, batching: bool = True, streams: bool = True,
        log=print) -> dict:
    import torch
    ctx, meta, nodes, nv = build(topology)
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
    drag = ctx.ib_get_forces(levels)[1]
    mass = [float(ctx.conservation(lv)[0]) for lv in range(levels + 1)]
    ctx.close()
    res = {"workload": "D3Q19 SRT + Smagorinsky (Cs 0.1) flow past a cube, "
                       f"coarse {'x'.join(str(v) for v in meta['n'])}, {levels} refinement levels "
                       f"({':'.join(str(1 << lv) for lv in range(levels + 1))} sub-cycling), inflow {U_IN}, convective outflow, "
                       f"Re {RE:.0f}, FP32, immersed-boundary cube ({nv} vertices)",
           "batched_level_steps": batching and not streams, "level_streams": streams, "cuda_graph": graph,
           "nodes_per_level": nodes, "lups_per_coarse_step": lups_per_step, "coarse_steps": steps,
           "ms_per_coarse_step": ms / steps, "mlups": lups_per_step * steps / (ms * 1e-3) / 1e6,
           "cube_force_total": [float(v) for v in drag], "mass_per_level": mass,
           "finite": bool(np.all(np.isfinite(mass)) and np.all(np.isfinite(drag)))}
    log(json.dumps(res))
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--topology", default=DEFAULT_TOPOLOGY)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--graph", type=int, default=1)
    ap.add_argument("--batching", type=int, default=1)
    ap.add_argument("--streams", type=int, default=1, help="per-level streams (zl_set_level_streams)")
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    run(a.topology, a.steps, a.warmup, bool(a.graph), bool(a.batching), bool(a.streams))
    print(f"wall {time.perf_counter() - t0:.1f} s")


if __name__ == "__main__":
    main()
