"""Generate the committed golden fixtures from the reference ZLLBM solver itself.

Run in a container that has the reference sources (the oracle harness
``oracle/_ref/zl_ref_run`` is built from them by ``make -C oracle ref``):

    python tests/golden/make_golden.py

Each ``lbm_<name>.npz`` holds the configuration, the Morton codes of every stored
node (reference order: sorted codes) and the populations before and after
``steps`` time steps of the reference's own TimeMarching.  ``morton_<d>d.npz``
holds codes and the reference's FindXNeg/FindXPos/... results for them.  ``vtu_<name>.npz``
holds the .vtu/.pvtu files the reference's own VTK writer produced after a run (binary and
ASCII), with each level's codes, flags, populations and node member rho_ at that time
(``python tests/golden/make_golden.py vtu`` regenerates only those).  ``amr_<name>.npz`` holds
multi-level and immersed-boundary runs with their interface layers and vertex records,
``ckpt_<name>.npz`` the reference's checkpoint files (``checkpoints``), ``ibpin_<name>.npz`` one
immersed-boundary step from a Taylor-Green field (``ibpin``), ``topo_*_small.npz`` small grids
refined around a body by the reference's grid builder (``topo``), and ``config_<name>.npz`` the
benchmark configurations at full length (``config``; ``c4`` regenerates only the cylinder's force
series); the word in brackets is the argument that regenerates only that group.  ``main`` (no
argument) regenerates every group but ``config``, which takes about half an hour of CPU time.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.port import (BC_BOUNCE_BACK, BC_NONEQ, BC_PERIODIC, MRT, REF_RUN, SRT, LevelConfig,  # noqa: E402
                         run_reference)

Z3 = (0.0, 0.0, 0.0)

CASES = {
    # lid-driven cavity (configuration of the small plain-method case at reduced size)
    "cavity2d_srt": (LevelConfig(dims=2, n=(16, 16), collision=SRT, nu=0.016,
                                 bc_kind=(BC_BOUNCE_BACK,) * 4 + (0, 0),
                                 bc_vel=(Z3, Z3, Z3, (0.1, 0.0, 0.0), Z3, Z3)), 200, "eq"),
    "cavity2d_mrt": (LevelConfig(dims=2, n=(16, 16), collision=MRT, nu=0.016,
                                 bc_kind=(BC_BOUNCE_BACK,) * 4 + (0, 0),
                                 bc_vel=(Z3, Z3, Z3, (0.1, 0.0, 0.0), Z3, Z3)), 200, "eq"),
    # periodic Taylor-Green vortex, 3D (MRT and SRT) and 2D
    "tgv3d_mrt": (LevelConfig(dims=3, n=(11, 11, 11), collision=MRT, nu=0.05 / 3.0,
                              bc_kind=(BC_PERIODIC,) * 6), 30, "tgv"),
    "tgv3d_srt": (LevelConfig(dims=3, n=(11, 11, 11), collision=SRT, nu=0.05 / 3.0,
                              bc_kind=(BC_PERIODIC,) * 6), 30, "tgv"),
    "tgv2d_mrt": (LevelConfig(dims=2, n=(17, 17), collision=MRT, nu=0.02,
                              bc_kind=(BC_PERIODIC,) * 4 + (0, 0)), 50, "tgv"),
    # channel: non-equilibrium extrapolation inflow/outflow, bounce-back walls
    "channel2d_neq": (LevelConfig(dims=2, n=(20, 12), collision=SRT, nu=0.05,
                                  bc_kind=(BC_NONEQ, BC_NONEQ, BC_BOUNCE_BACK, BC_BOUNCE_BACK, 0, 0),
                                  bc_vel=((0.05, 0, 0), (0.05, 0, 0), Z3, Z3, Z3, Z3)), 60, "eq"),
    # mixed faces in 3D: NEQ in x, moving-wall bounce-back in y, periodic z
    "box3d_mixed": (LevelConfig(dims=3, n=(10, 8, 9), collision=MRT, nu=0.05,
                                bc_kind=(BC_NONEQ, BC_NONEQ, BC_BOUNCE_BACK, BC_BOUNCE_BACK, BC_PERIODIC, BC_PERIODIC),
                                bc_vel=((0.05, 0, 0), (0.05, 0, 0), Z3, (0.03, 0, 0.01), Z3, Z3)), 30, "eq"),
    # bounce back with moving walls next to a periodic axis (device wraps the periodic axis)
    "box3d_bbper": (LevelConfig(dims=3, n=(9, 10, 8), collision=SRT, nu=0.04,
                                bc_kind=(BC_BOUNCE_BACK, BC_BOUNCE_BACK, BC_BOUNCE_BACK, BC_BOUNCE_BACK,
                                         BC_PERIODIC, BC_PERIODIC),
                                bc_vel=((0, 0.02, 0), Z3, Z3, (0.05, 0, 0.02), Z3, Z3)), 40, "eq"),
    "channel2d_per": (LevelConfig(dims=2, n=(14, 11), collision=MRT, nu=0.03,
                                  bc_kind=(BC_PERIODIC, BC_PERIODIC, BC_BOUNCE_BACK, BC_BOUNCE_BACK, 0, 0),
                                  bc_vel=(Z3, Z3, Z3, (0.08, 0, 0), Z3, Z3)), 80, "eq"),
}


# multi-level grids refined around a default shape (the reference's GeometryInfoOrigin), NEQ inflow/outflow
AMR_CASES = {
    "amr2d_l1": dict(dims=2, n=(40, 32), levels=1, geo="circle:20,16,3", ext=3, inner=2, coll="srt", nu=0.02,
                     bc=["xmin:neq:0.05,0", "xmax:neq:0.05,0", "ymin:bb", "ymax:bb"], steps=6),
    "amr2d_l2": dict(dims=2, n=(48, 40), levels=2, geo="circle:24,20,2", ext=3, inner=2, coll="mrt", nu=0.01,
                     bc=["xmin:neq:0.04,0", "xmax:neq:0.04,0", "ymin:bb", "ymax:bb:0.02,0"], steps=4),
    "amr3d_l1": dict(dims=3, n=(20, 16, 16), levels=1, geo="cube:10,8,8,2", ext=2, inner=1, coll="mrt", nu=0.02,
                     bc=["xmin:neq:0.05,0,0", "xmax:neq:0.05,0,0", "ymin:bb", "ymax:bb", "zmin:bb", "zmax:bb"], steps=3),
}


# immersed boundary (reference GeometryInfoImmersedBoundary, direct forcing every sub-step of its level)
AMR_CASES.update({
    "ib2d_l0": dict(dims=2, n=(40, 32), levels=0, ib="circle:20.5,16.5,3", ext=3, inner=2, coll="srt", nu=0.02,
                    bc=["xmin:neq:0.05,0", "xmax:neq:0.05,0", "ymin:bb", "ymax:bb"], steps=8),
    "ib2d_l1": dict(dims=2, n=(48, 40), levels=1, ib="circle:24.3,20.1,2.5", ext=3, inner=2, coll="mrt", nu=0.01,
                    bc=["xmin:neq:0.04,0", "xmax:neq:0.04,0", "ymin:bb", "ymax:bb"], steps=4),
    "ib3d_l0": dict(dims=3, n=(20, 16, 16), levels=0, ib="sphere:10.2,8.1,7.9,2.5", ext=2, inner=1, coll="srt",
                    nu=0.03, bc=["xmin:neq:0.05,0,0", "xmax:neq:0.05,0,0", "ymin:bb", "ymax:bb", "zmin:bb", "zmax:bb"],
                    steps=4),
    # constant body force (SetConstantForce), periodic channel
    "force2d_mrt": dict(dims=2, n=(12, 10), levels=0, coll="mrt", nu=0.05, cforce="1e-4,2e-5",
                        bc=["xmin:per", "xmax:per", "ymin:bb", "ymax:bb"], steps=40),
    "force3d_srt": dict(dims=3, n=(8, 9, 7), levels=0, coll="srt", nu=0.05, cforce="1e-4,0,-3e-5",
                        bc=["xmin:per", "xmax:per", "ymin:bb", "ymax:bb", "zmin:per", "zmax:per"], steps=30),
})


# one step of the reference's direct forcing from a non-uniform (Taylor-Green) velocity field, to
# pin the oracle's interpolation: the vertex forces after the step are those of the first pass,
# which reads the initial populations
IB_PIN_CASES = {
    "ib2d": dict(dims=2, n=(40, 32), levels=0, ib="circle:20.5,16.5,3", ext=3, inner=2, coll="srt", nu=0.02,
                 bc=["xmin:per", "xmax:per", "ymin:per", "ymax:per"], steps=1, init="tgv", u0=0.05),
    "ib3d": dict(dims=3, n=(20, 16, 16), levels=0, ib="sphere:10.2,8.1,7.9,2.5", ext=2, inner=1, coll="srt",
                 nu=0.03, bc=["xmin:per", "xmax:per", "ymin:per", "ymax:per", "zmin:per", "zmax:per"], steps=1,
                 init="tgv", u0=0.05),
}


def run_amr(name, case, tmp, prefix="amr"):
    from oracle.port import load_levels
    wd = os.path.join(tmp, name)
    os.makedirs(wd, exist_ok=True)
    args = [REF_RUN, f"dims={case['dims']}", "n=" + ",".join(str(v) for v in case["n"]), f"levels={case['levels']}",
            f"coll={case['coll']}", f"nu={case['nu']!r}", f"steps={case['steps']}",
            "lout0=" + os.path.join(wd, "l0.bin"), "lout=" + os.path.join(wd, "l1.bin")] + \
           [f"bc={b}" for b in case["bc"]]
    for key in ("geo", "ib", "ext", "inner", "cforce", "init", "u0"):
        if key in case:
            args.append(f"{key}={case[key]}")
    if "ib" in case:
        args += ["vout0=" + os.path.join(wd, "v0.bin"), "vout=" + os.path.join(wd, "v1.bin")]
    if "cforce" in case:
        args.append("forces=1")
    subprocess.run(args, check=True, cwd=wd, stdout=subprocess.DEVNULL)
    dims, q, before = load_levels(os.path.join(wd, "l0.bin"))
    _, _, after = load_levels(os.path.join(wd, "l1.bin"))
    out = {"meta": json.dumps(case)}
    for lv, (b, a) in enumerate(zip(before, after)):
        assert np.array_equal(b["nodes"]["code"], a["nodes"]["code"])
        out[f"codes{lv}"] = b["nodes"]["code"]
        out[f"flags{lv}"] = b["nodes"]["flag"]
        out[f"f_before{lv}"] = b["nodes"]["f"]
        out[f"f_after{lv}"] = a["nodes"]["f"]
        lay = b["layers"]
        empty = np.zeros(0, dtype=np.uint64)
        out[f"c2f_fine{lv}"] = np.union1d(np.union1d(lay.get((2, 1), empty), lay.get((3, 1), empty)),
                                          np.union1d(lay.get((2, 2), empty), lay.get((3, 2), empty)))
        out[f"f2c_coarse{lv}"] = np.union1d(lay.get((0, 1), empty), lay.get((1, 1), empty))
    if "ib" in case:
        for tag, fn in (("before", "v0.bin"), ("after", "v1.bin")):
            raw = open(os.path.join(wd, fn), "rb").read()
            nv = int(np.frombuffer(raw[:8], np.int64)[0])
            out[f"vertices_{tag}"] = np.frombuffer(raw[8:], np.float64, count=nv * 10).reshape(nv, 10)
    np.savez_compressed(os.path.join(HERE, f"{prefix}_{name}.npz"), **out)
    print(name, [len(l["nodes"]) for l in before], "nodes per level")


# checkpoints written by the reference's own writer (IoManager::WriteCheckPointData) after a run
CKPT_CASES = ("amr2d_l1", "amr3d_l1", "force2d_mrt", "force3d_srt")


def run_checkpoint(name, case, tmp):
    """grid_nodes of the reference's checkpoint folder and every level's state at that time."""
    from oracle.port import load_levels
    wd = os.path.join(tmp, "ckpt_" + name)
    os.makedirs(wd, exist_ok=True)
    args = [REF_RUN, f"dims={case['dims']}", "n=" + ",".join(str(v) for v in case["n"]), f"levels={case['levels']}",
            f"coll={case['coll']}", f"nu={case['nu']!r}", f"steps={case['steps']}",
            "lout=" + os.path.join(wd, "l1.bin"), "ckpt=" + os.path.join(wd, "run")] + [f"bc={b}" for b in case["bc"]]
    for key in ("geo", "ib", "ext", "inner", "cforce"):
        if key in case:
            args.append(f"{key}={case[key]}")
    if "cforce" in case:
        args.append("forces=1")
    subprocess.run(args, check=True, cwd=wd, stdout=subprocess.DEVNULL)
    _, _, after = load_levels(os.path.join(wd, "l1.bin"))
    raw = np.fromfile(os.path.join(wd, f"run_checkpoint{case['steps']}", "grid_nodes"), np.uint8)
    out = {"meta": json.dumps(case), "grid_nodes": raw}
    for lv, a in enumerate(after):
        out[f"codes{lv}"] = a["nodes"]["code"]
        out[f"flags{lv}"] = a["nodes"]["flag"]
        out[f"f{lv}"] = a["nodes"]["f"]
    np.savez_compressed(os.path.join(HERE, f"ckpt_{name}.npz"), **out)
    print("checkpoint", name, raw.size, "bytes")


# field output written by the reference's own VTK writer (IoManager::OutputMeshData) after a run
VTU_CASES = {
    "tgv3d": dict(dims=3, n=(4, 4, 4), levels=0, coll="mrt", nu=0.02, init="tgv", u0=0.05,
                  bc=["xmin:per", "xmax:per", "ymin:per", "ymax:per", "zmin:per", "zmax:per"], steps=3),
    "amr2d_l1": dict(AMR_CASES["amr2d_l1"], steps=2),
    "force2d_mrt": dict(AMR_CASES["force2d_mrt"], steps=5),
}


def run_vtu(name, case, tmp):
    """The reference's .vtu/.pvtu text (binary and ASCII) with every level's state at that time."""
    from oracle.port import load_levels
    out = {"meta": json.dumps(case)}
    for binary in (1, 0):
        wd = os.path.join(tmp, f"vtu_{name}_{binary}")
        os.makedirs(wd, exist_ok=True)
        args = [REF_RUN, f"dims={case['dims']}", "n=" + ",".join(str(v) for v in case["n"]),
                f"levels={case['levels']}", f"coll={case['coll']}", f"nu={case['nu']!r}", f"steps={case['steps']}",
                "lout=" + os.path.join(wd, "l1.bin"), "rout=" + os.path.join(wd, "rho.bin"),
                "vtu=" + os.path.join(wd, "run"), f"vtu_binary={binary}"] + [f"bc={b}" for b in case["bc"]]
        for key in ("geo", "ib", "ext", "inner", "cforce", "init", "u0"):
            if key in case:
                args.append(f"{key}={case[key]}")
        if "cforce" in case:
            args.append("forces=1")
        subprocess.run(args, check=True, cwd=wd, stdout=subprocess.DEVNULL)
        tag = "bin" if binary else "asc"
        folder = os.path.join(wd, "run_data")
        levels = case["levels"] + 1
        for lv in range(levels):
            out[f"vtu_{tag}{lv}"] = np.fromfile(os.path.join(folder, f"rank_0_grid_level_{lv}.vtu"), np.uint8)
        out[f"pvtu_{tag}"] = np.fromfile(os.path.join(folder, "rank_0_.pvtu"), np.uint8)
        if binary:
            _, _, after = load_levels(os.path.join(wd, "l1.bin"))
            raw = open(os.path.join(wd, "rho.bin"), "rb").read()
            pos = 4
            for lv, a in enumerate(after):
                out[f"codes{lv}"] = a["nodes"]["code"]
                out[f"flags{lv}"] = a["nodes"]["flag"]
                out[f"f{lv}"] = a["nodes"]["f"]
                nr = int(np.frombuffer(raw[pos:pos + 8], np.int64)[0])
                rec = np.frombuffer(raw[pos + 8:pos + 8 + nr * 16], dtype=[("code", "<u8"), ("rho", "<f8")])
                assert np.array_equal(rec["code"], a["nodes"]["code"])
                out[f"rho_member{lv}"] = rec["rho"].copy()
                pos += 8 + nr * 16
    np.savez_compressed(os.path.join(HERE, f"vtu_{name}.npz"), **out)
    print("vtu", name, [out[f"vtu_bin{lv}"].size for lv in range(case["levels"] + 1)], "bytes (binary)")


def morton_cases(dims: int, rng: np.random.Generator) -> np.ndarray:
    nb = 64 // dims
    edge = []
    for a in range(dims):
        for v in (0, 1, 2, (1 << nb) - 1, (1 << nb) - 2, 1 << (nb - 1)):
            idx = [5] * dims
            idx[a] = v
            code = 0
            for i in range(nb):
                for b in range(dims):
                    code |= ((idx[b] >> i) & 1) << (dims * i + b)
            edge.append(code)
    edge += [0, (1 << 64) - 1, 1 << 63, (1 << 63) - 1]
    rand = rng.integers(0, 2**63, size=200, dtype=np.int64).astype(np.uint64) * np.uint64(2) + \
        rng.integers(0, 2, size=200, dtype=np.int64).astype(np.uint64)
    return np.concatenate([np.array(edge, dtype=np.uint64), rand])


def main():
    if not os.path.exists(REF_RUN):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    with tempfile.TemporaryDirectory() as tmp:
        for name, (cfg, steps, init) in CASES.items():
            before, after = run_reference(cfg, steps, os.path.join(tmp, name), init=init, u0=0.05)
            assert np.array_equal(before["code"], after["code"])
            meta = dict(dims=cfg.dims, n=list(cfg.n), collision=cfg.collision, nu=cfg.nu, rho0=cfg.rho0,
                        bc_kind=list(cfg.bc_kind), bc_vel=[list(v) for v in cfg.bc_vel], steps=steps, init=init,
                        u0=0.05)
            np.savez_compressed(os.path.join(HERE, f"lbm_{name}.npz"), meta=json.dumps(meta),
                                codes=before["code"], f_before=before["f"], f_after=after["f"])
            print(name, before.size, "nodes")
        for name, case in AMR_CASES.items():
            run_amr(name, case, tmp)
        run_ib_pins(tmp)
        for name in CKPT_CASES:
            run_checkpoint(name, AMR_CASES[name], tmp)
        for name, case in VTU_CASES.items():
            run_vtu(name, case, tmp)
        for dims in (2, 3):
            fout = os.path.join(tmp, f"les{dims}.bin")
            subprocess.run([REF_RUN, "mode=les", f"dims={dims}", f"out={fout}"], check=True, cwd=tmp,
                           stdout=subprocess.DEVNULL)
            q = 9 if dims == 2 else 19
            np.savez_compressed(os.path.join(HERE, f"les_{dims}d.npz"),
                                records=np.fromfile(fout, np.float64).reshape(-1, 2 + 2 * q + 3 + 3 + 2))
            print("les", dims)
        rng = np.random.default_rng(20261203)
        for dims in (2, 3):
            codes = morton_cases(dims, rng)
            fin = os.path.join(tmp, f"codes{dims}.bin")
            fout = os.path.join(tmp, f"nbr{dims}.bin")
            codes.tofile(fin)
            subprocess.run([REF_RUN, "mode=morton", f"dims={dims}", f"in={fin}", f"out={fout}"], check=True,
                           cwd=tmp, stdout=subprocess.DEVNULL)
            nbr = np.fromfile(fout, dtype=np.uint64).reshape(codes.size, 2 * dims)
            np.savez_compressed(os.path.join(HERE, f"morton_{dims}d.npz"), codes=codes, neighbors=nbr)
            print("morton", dims, codes.size)
    run_topologies()


# small grids refined around a body (the reference's own grid builder) for the multi-level flow drivers
TOPO_CASES = {
    "topo_cube_small": ["--n", "48,32,32", "--levels", "2", "--cube", "16,16,16,4", "--ext", "2", "--inner", "4"],
    "topo_cylinder_small": ["--n", "96,48", "--levels", "2", "--circle", "24,24,1.5", "--ext", "3", "--inner", "3"],
}


def run_topologies():
    for name, args in TOPO_CASES.items():
        subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "make_body_topology.py"),
                        os.path.join(HERE, f"{name}.npz")] + args, check=True)


def run_ib_pins(tmp):
    for name, case in IB_PIN_CASES.items():
        run_amr(name, case, tmp, prefix="ibpin")


# the benchmark configurations at full length (``config``): the 256^2 cavity of the plain method
# (20,000 steps) and the D3Q19 MRT Taylor-Green vortex at 64^3 (5,000 steps).  The populations
# after the run are kept as a SHA-256 of their bytes (sorted codes, float64 little endian) for the
# bit-exact FP64 check, plus the reference's output velocity (cavity: the whole field; TGV: the
# kinetic energy and one x-line), recomputed from f_ as its output rule does.
CONFIG_CASES = {
    "c1_cavity256": (LevelConfig(dims=2, n=(256, 256), collision=SRT, nu=0.1 * 256 / 100,
                                 bc_kind=(BC_BOUNCE_BACK,) * 4 + (0, 0),
                                 bc_vel=(Z3, Z3, Z3, (0.1, 0.0, 0.0), Z3, Z3)), 20000, "eq"),
    "c2_tgv64": (LevelConfig(dims=3, n=(65, 65, 65), collision=MRT, nu=0.05 / 3.0,
                             bc_kind=(BC_PERIODIC,) * 6), 5000, "tgv"),
}

# the immersed-boundary cylinder of the D2Q9 MRT configuration, reduced: 4 levels on a 128 x 64
# coarse domain (the full case's 1024 x 512 divided by 8 per axis), diameter 40 finest cells,
# inflow 0.04, Re 200 (nu = 0.04 * 5 / 200 at the background level), every node starting at
# feq(1, (0.04, 0)) so that the body is loaded from the first step; 200 background steps
# (1,600 finest steps).  Kept: each level's codes, flags and interface layers, the vertices, and
# the force sum F area after every background step.
C4_CASE = dict(dims=2, n=(128, 64), levels=3, ib="circle:40.3,32.1,2.5", ext=3, inner=2, coll="mrt",
               nu=0.04 * 5 / 200, vel="0.04,0", bc=["xmin:neq:0.04,0", "xmax:neq:0.04,0", "ymin:bb", "ymax:bb"],
               steps=200)


def output_velocity(f, dims):
    """The reference's output velocity: recomputed from f_ (lbm_grid_interface.cpp:614-657)."""
    from oracle.port import LATTICE_C
    c = np.array(LATTICE_C[dims], dtype=np.float64)
    return (f @ c) / f.sum(1)[:, None]


def run_configs(tmp):
    import hashlib
    for name, (cfg, steps, init) in CONFIG_CASES.items():
        before, after = run_reference(cfg, steps, os.path.join(tmp, name), init=init, u0=0.05)
        assert np.array_equal(before["code"], after["code"])
        f = np.ascontiguousarray(after["f"], dtype="<f8")
        meta = dict(dims=cfg.dims, n=list(cfg.n), collision=cfg.collision, nu=cfg.nu, rho0=cfg.rho0,
                    bc_kind=list(cfg.bc_kind), bc_vel=[list(v) for v in cfg.bc_vel], steps=steps, init=init,
                    u0=0.05, f_after_sha256=hashlib.sha256(f.tobytes()).hexdigest())
        u = output_velocity(f, cfg.dims)
        out = dict(meta=json.dumps(meta), codes=before["code"])
        if cfg.dims == 2:
            out["velocity_after"] = u
        else:
            from oracle.port import morton_decode
            idx = morton_decode(before["code"], cfg.dims) - 1
            line = (idx[:, 1] == cfg.n[1] // 4) & (idx[:, 2] == cfg.n[2] // 4)
            order = np.argsort(idx[line, 0])
            out["line_codes"] = before["code"][line][order]
            out["line_velocity"] = u[line][order]
            rho = f.sum(1)
            out["kinetic_energy"] = np.array(0.5 * (rho * (u * u).sum(1)).sum())
        np.savez_compressed(os.path.join(HERE, f"config_{name}.npz"), **out)
        print(name, before.size, "nodes", steps, "steps")
    run_c4(tmp)


def run_c4(tmp):
    from oracle.port import load_levels
    case = C4_CASE
    wd = os.path.join(tmp, "c4")
    os.makedirs(wd, exist_ok=True)
    args = [REF_RUN, f"dims={case['dims']}", "n=" + ",".join(str(v) for v in case["n"]), f"levels={case['levels']}",
            f"coll={case['coll']}", f"nu={case['nu']!r}", f"steps={case['steps']}", f"vel={case['vel']}",
            f"ib={case['ib']}", f"ext={case['ext']}", f"inner={case['inner']}",
            "lout0=" + os.path.join(wd, "l0.bin"), "vout0=" + os.path.join(wd, "v0.bin"),
            "vout=" + os.path.join(wd, "v1.bin"), "fhist=" + os.path.join(wd, "fh.bin")] + \
           [f"bc={b}" for b in case["bc"]]
    subprocess.run(args, check=True, cwd=wd, stdout=subprocess.DEVNULL)
    dims, q, before = load_levels(os.path.join(wd, "l0.bin"))
    out = {"meta": json.dumps(case)}
    for lv, b in enumerate(before):
        out[f"codes{lv}"] = b["nodes"]["code"]
        out[f"flags{lv}"] = b["nodes"]["flag"]
        lay = b["layers"]
        empty = np.zeros(0, dtype=np.uint64)
        out[f"c2f_fine{lv}"] = np.union1d(np.union1d(lay.get((2, 1), empty), lay.get((3, 1), empty)),
                                          np.union1d(lay.get((2, 2), empty), lay.get((3, 2), empty)))
        out[f"f2c_coarse{lv}"] = np.union1d(lay.get((0, 1), empty), lay.get((1, 1), empty))
        # every node starts at the same equilibrium: keep one node's populations
        f0 = b["nodes"]["f"]
        assert np.array_equal(f0, np.broadcast_to(f0[0], f0.shape))
        out[f"f_init{lv}"] = f0[0].copy()
    for tag, fn in (("before", "v0.bin"), ("after", "v1.bin")):
        raw = open(os.path.join(wd, fn), "rb").read()
        nv = int(np.frombuffer(raw[:8], np.int64)[0])
        out[f"vertices_{tag}"] = np.frombuffer(raw[8:], np.float64, count=nv * 10).reshape(nv, 10)
    raw = open(os.path.join(wd, "fh.bin"), "rb").read()
    nh = int(np.frombuffer(raw[:8], np.int64)[0])
    out["force_history"] = np.frombuffer(raw[8:], np.float64, count=nh * 3).reshape(nh, 3)
    np.savez_compressed(os.path.join(HERE, "config_c4_cylinder_reduced.npz"), **out)
    print("c4", [len(l["nodes"]) for l in before], "nodes per level,", nh, "force samples")


if __name__ == "__main__":
    if sys.argv[1:] == ["topo"]:
        run_topologies()
    elif sys.argv[1:] == ["config"]:
        if not os.path.exists(REF_RUN):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
        with tempfile.TemporaryDirectory() as tmp:
            run_configs(tmp)
    elif sys.argv[1:] == ["c4"]:
        with tempfile.TemporaryDirectory() as tmp:
            run_c4(tmp)
    elif sys.argv[1:] == ["ibpin"]:
        if not os.path.exists(REF_RUN):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
        with tempfile.TemporaryDirectory() as tmp:
            run_ib_pins(tmp)
    elif sys.argv[1:] == ["vtu"]:
        if not os.path.exists(REF_RUN):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
        with tempfile.TemporaryDirectory() as tmp:
            for name, case in VTU_CASES.items():
                run_vtu(name, case, tmp)
    elif sys.argv[1:] == ["checkpoints"]:
        if not os.path.exists(REF_RUN):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
        with tempfile.TemporaryDirectory() as tmp:
            for name in CKPT_CASES:
                run_checkpoint(name, AMR_CASES[name], tmp)
    else:
        main()
