"""Loading the golden fixtures and mapping them onto the oracle and the C ABI."""
from __future__ import annotations

import glob
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def lbm_fixture_names() -> list[str]:
    return sorted(os.path.basename(p)[4:-4] for p in glob.glob(os.path.join(GOLDEN, "lbm_*.npz")))


def load_lbm(name: str):
    z = np.load(os.path.join(GOLDEN, f"lbm_{name}.npz"))
    meta = json.loads(str(z["meta"]))
    return meta, z["codes"], z["f_before"], z["f_after"]


def level_config(meta):
    from oracle.port import LevelConfig
    return LevelConfig(dims=meta["dims"], n=tuple(meta["n"]), collision=meta["collision"], nu=meta["nu"],
                       rho0=meta["rho0"], bc_kind=tuple(meta["bc_kind"]), bc_vel=tuple(tuple(v) for v in meta["bc_vel"]))


def solver_config(meta, storage: int):
    import zllbm_b200 as zl
    dims = meta["dims"]
    n = list(meta["n"]) + [1] * (3 - dims)
    return zl.SolverConfig(
        lattice=zl.D2Q9 if dims == 2 else zl.D3Q19, collision=meta["collision"], storage=storage,
        viscosity=meta["nu"], rho0=meta["rho0"], bc_kind=tuple(meta["bc_kind"]),
        bc_velocity=tuple(tuple(v) for v in meta["bc_vel"]),
        domain_min=(1, 1, 1 if dims == 3 else 0), domain_max=(n[0], n[1], n[2] if dims == 3 else 0))


def grid_order(codes, dims, n):
    """Permutation taking dump order (sorted codes) to the oracle's x-fastest grid order."""
    from oracle.port import morton_decode
    idx = morton_decode(codes, dims) - 1
    lin = idx[:, 0] + n[0] * idx[:, 1]
    if dims == 3:
        lin = lin + n[0] * n[1] * idx[:, 2]
    return lin
