"""Build the zllbm_b200 CUDA library (sm_100a) in-tree.

    python -m zllbm_b200.build          # -> zllbm_b200/libzllbm_b200.so

Each translation unit is compiled with nvcc for sm_100a only; the FP64 kernels
are built with -fmad=false so their arithmetic follows the reference's
rounding step for step.  Objects go to zllbm_b200/_build/.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libzllbm_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC]

SOURCES = {
    "api.cu": [],
    "topology.cu": [],
    "kernels_f64.cu": ["-fmad=false"],
    "kernels_f32.cu": [],
    "kernels_f16.cu": [],
    "static_scratch.cu": [],
    "closure.cu": [],
    "vtu.cu": [],
}

# The fused step and batched step kernels, one translation unit per (storage, lattice, collision,
# part) so that they compile in parallel: (object stem, storage type, extra flags).
STEP_STORAGES = [("f64", "double", ["-fmad=false"]), ("f32", "float", []),
                 ("f16", "__half", []), ("bf16", "__nv_bfloat16", [])]
STEP_LATTICES = [("d2q9", "zl::D2Q9"), ("d3q19", "zl::D3Q19")]
STEP_COLLISIONS = [("srt", "zl::kSrt"), ("mrt", "zl::kMrt")]
# even / odd step, then the batched step with no extension, force, LES, force + LES
STEP_PARTS = ["even", "odd", "batch", "batch_force", "batch_les", "batch_force_les"]


def units() -> list[tuple[str, str, list[str]]]:
    """(source, object, flags) of every translation unit of the library."""
    out = []
    step_src = os.path.join(CSRC, "step_inst.cu")
    for st, ty, flags in STEP_STORAGES:
        for lt, lty in STEP_LATTICES:
            for ct, cty in STEP_COLLISIONS:
                for part, name in enumerate(STEP_PARTS):
                    defs = [f"-DZL_STEP_S={ty}", f"-DZL_STEP_L={lty}", f"-DZL_STEP_C={cty}", f"-DZL_STEP_PART={part}"]
                    out.append((step_src, os.path.join(BUILD, f"step_{st}_{lt}_{ct}_{name}.o"), flags + defs))
    # the step units are the longest compiles: they come first in the job list
    out += [(os.path.join(CSRC, src), os.path.join(BUILD, src.replace(".cu", ".o")), flags)
            for src, flags in SOURCES.items()]
    return out


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _deps(obj: str) -> list[str] | None:
    """Files the object was built from, read from the dependency file nvcc wrote beside it."""
    d = obj[:-2] + ".d"
    if not os.path.exists(d):
        return None
    text = open(d).read().replace("\\\n", " ")
    _, _, rest = text.partition(":")
    return rest.split()


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(not os.path.exists(d) or os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    jobs = []
    for src, obj, flags in units():
        objs.append(obj)
        deps = _deps(obj)
        if deps is None or _stale(obj, deps + [src, __file__]):
            cmd = ([nvcc()] + ARCH + COMMON + flags + (extra or []) +
                   ["-MD", "-MF", obj[:-2] + ".d", "-c", src, "-o", obj])
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr)

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    if jobs or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        run(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None))
