"""ORACLE — test infrastructure only.

Python helpers around the CPU oracle:

* ``load_dump`` reads the binary node dumps written by ``oracle/ref_harness.cpp``
  (the reference ZLLBM solver driven through its own API);
* ``morton_decode`` turns the reference's Morton codes back into integer indices
  (restates ``SFBitsetComputeIndices``, amr_project/grid/morton_aux.cpp:107-119 and
  :336-351);
* ``Port`` wraps the C restatement ``oracle/zl_port.c`` through ctypes.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may use this module, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
PORT_SO = os.path.join(REF_DIR, "libzl_port.so")
REF_RUN = os.path.join(REF_DIR, "zl_ref_run")

BC_NONE, BC_BOUNCE_BACK, BC_PERIODIC, BC_NONEQ = 0, 1, 2, 3
BC_CONVECTIVE = 4  # not in the reference; restated in zl_port.c
SRT, MRT = 0, 1
FACES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


def load_dump(path: str):
    """Return (dims, q, records) for a reference dump; records has fields code, flag, f."""
    with open(path, "rb") as fh:
        raw = fh.read()
    dims, q = np.frombuffer(raw[:8], np.int32)
    n = int(np.frombuffer(raw[8:16], np.int64)[0])
    rec = np.dtype([("code", "<u8"), ("flag", "<i4"), ("pad", "<i4"), ("f", "<f8", (int(q),))])
    return int(dims), int(q), np.frombuffer(raw[16:], rec, count=n)


def morton_decode(codes: np.ndarray, dims: int) -> np.ndarray:
    """Per-axis integer indices of interleaved Morton codes (x at bit dims*i, y at dims*i+1, ...)."""
    codes = np.asarray(codes, dtype=np.uint64)
    out = np.zeros((codes.size, dims), dtype=np.int64)
    nbits = 64 // dims
    for i in range(nbits):
        for a in range(dims):
            bit = (codes >> np.uint64(dims * i + a)) & np.uint64(1)
            out[:, a] |= bit.astype(np.int64) << i
    return out


def morton_encode(idx: np.ndarray, dims: int) -> np.ndarray:
    """Inverse of ``morton_decode`` (restates SFBitsetEncoding, morton_aux.cpp:53-63, :274-286)."""
    idx = np.asarray(idx, dtype=np.uint64).reshape(-1, dims)
    out = np.zeros(idx.shape[0], dtype=np.uint64)
    nbits = 64 // dims
    for i in range(nbits):
        for a in range(dims):
            bit = (idx[:, a] >> np.uint64(i)) & np.uint64(1)
            out |= bit << np.uint64(dims * i + a)
    return out


def dump_to_grid(records, dims: int, n_nodes) -> np.ndarray:
    """Scatter dump records into an x-fastest array f[z, y, x, q] (reference index - 1 = grid index)."""
    idx = morton_decode(records["code"], dims) - 1
    q = records["f"].shape[1]
    shape = tuple(reversed(n_nodes[:dims])) + (q,)
    grid = np.full(shape, np.nan)
    if dims == 2:
        grid[idx[:, 1], idx[:, 0]] = records["f"]
    else:
        grid[idx[:, 2], idx[:, 1], idx[:, 0]] = records["f"]
    return grid


class ZlpLevel(ctypes.Structure):
    _fields_ = [
        ("dims", ctypes.c_int),
        ("n", ctypes.c_int * 3),
        ("collision", ctypes.c_int),
        ("level", ctypes.c_int),
        ("nu", ctypes.c_double),
        ("rho0", ctypes.c_double),
        ("bc_kind", ctypes.c_int * 6),
        ("bc_vel", (ctypes.c_double * 3) * 6),
        ("les", ctypes.c_int),
        ("les_cs", ctypes.c_double),
        ("has_force", ctypes.c_int),
        ("force", ctypes.c_double * 3),
        ("node_force", ctypes.POINTER(ctypes.c_double)),
    ]


@dataclass
class LevelConfig:
    """One uniform level in the reference's stored-node convention (n = cells + 1)."""

    dims: int
    n: tuple
    collision: int = SRT
    nu: float = 0.1
    rho0: float = 1.0
    level: int = 0
    bc_kind: tuple = (0, 0, 0, 0, 0, 0)
    bc_vel: tuple = ((0.0, 0.0, 0.0),) * 6
    les: int = 0
    les_cs: float = 0.16
    force: tuple | None = None
    node_force: np.ndarray | None = None  # (nodes, 3) float64 in grid order, added to `force`
    extra: dict = field(default_factory=dict)

    @property
    def q(self) -> int:
        return 9 if self.dims == 2 else 19

    def to_c(self) -> ZlpLevel:
        c = ZlpLevel()
        c.dims = self.dims
        n = list(self.n) + [1] * (3 - len(self.n))
        for i in range(3):
            c.n[i] = int(n[i])
        c.collision = self.collision
        c.level = self.level
        c.nu = self.nu
        c.rho0 = self.rho0
        for i in range(6):
            c.bc_kind[i] = int(self.bc_kind[i])
            for a in range(3):
                c.bc_vel[i][a] = float(self.bc_vel[i][a]) if a < len(self.bc_vel[i]) else 0.0
        c.les = self.les
        c.les_cs = self.les_cs
        c.has_force = 1 if self.force is not None else 0
        if self.force is not None:
            for a in range(len(self.force)):
                c.force[a] = float(self.force[a])
        if self.node_force is not None:
            nf = self.node_force
            assert nf.dtype == np.float64 and nf.flags.c_contiguous and nf.shape[-1] == 3
            c.node_force = nf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        return c

    def harness_args(self) -> list:
        """Command-line for ``zl_ref_run`` describing the same level."""
        cells = ",".join(str(v - 1) for v in self.n[: self.dims])
        args = [f"dims={self.dims}", f"n={cells}", f"coll={'mrt' if self.collision == MRT else 'srt'}",
                f"nu={self.nu!r}", f"rho0={self.rho0!r}"]
        kinds = {BC_BOUNCE_BACK: "bb", BC_PERIODIC: "per", BC_NONEQ: "neq"}
        for i, face in enumerate(FACES[: 2 * self.dims]):
            k = self.bc_kind[i]
            if k:
                vel = ",".join(repr(float(v)) for v in self.bc_vel[i][: self.dims])
                args.append(f"bc={face}:{kinds[k]}:{vel}")
        return args


def build_port() -> str:
    """Compile the C restatement (strict IEEE flags) into oracle/_ref/libzl_port.so."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    return PORT_SO


class Port:
    """ctypes wrapper over oracle/zl_port.c."""

    def __init__(self, path: str = PORT_SO):
        if not os.path.exists(path):
            build_port()
        self.lib = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        self.lib.zlp_run.argtypes = [ctypes.POINTER(ZlpLevel), dp, dp, ctypes.c_int]
        self.lib.zlp_run.restype = ctypes.c_int
        self.lib.zlp_macros.argtypes = [ctypes.POINTER(ZlpLevel), dp, dp, dp]
        self.lib.zlp_feq.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp]
        self.lib.zlp_mrt_matrix.argtypes = [ctypes.c_int, ctypes.c_double, dp]
        self.lib.zlp_tau.argtypes = [ctypes.c_double, ctypes.c_int]
        self.lib.zlp_tau.restype = ctypes.c_double
        self.lib.zlp_smag_tau_sgs.argtypes = [ctypes.c_int, dp, dp, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_double, ctypes.c_int, dp, dp]
        self.lib.zlp_smag_tau_sgs.restype = ctypes.c_double

    @staticmethod
    def _ptr(a: np.ndarray):
        assert a.dtype == np.float64 and a.flags.c_contiguous
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    def run(self, cfg: LevelConfig, f: np.ndarray, fc: np.ndarray | None = None, steps: int = 1):
        """Advance in place; f (and fc) are [..., q] arrays in x-fastest node order."""
        if fc is None:
            fc = f.copy()
        c = cfg.to_c()
        rc = self.lib.zlp_run(ctypes.byref(c), self._ptr(f), self._ptr(fc), int(steps))
        if rc != 0:
            raise RuntimeError(f"zlp_run failed: {rc}")
        return f, fc

    def macros(self, cfg: LevelConfig, f: np.ndarray):
        nn = f.size // cfg.q
        rho = np.empty(nn)
        u = np.empty(nn * cfg.dims)
        self.lib.zlp_macros(ctypes.byref(cfg.to_c()), self._ptr(f), self._ptr(rho), self._ptr(u))
        return rho, u.reshape(nn, cfg.dims)

    def feq(self, dims: int, rho: float, u) -> np.ndarray:
        q = 9 if dims == 2 else 19
        uu = np.zeros(3)
        uu[: len(u)] = u
        out = np.empty(q)
        self.lib.zlp_feq(dims, rho, self._ptr(uu), self._ptr(out))
        return out

    def mrt_matrix(self, dims: int, tau: float) -> np.ndarray:
        q = 9 if dims == 2 else 19
        out = np.empty(q * q)
        self.lib.zlp_mrt_matrix(dims, tau, self._ptr(out))
        return out.reshape(q, q)

    def smag_tau_sgs(self, dims, f, feq, tau0, dt, cs, force=None, u=None) -> float:
        f, feq = np.ascontiguousarray(f, dtype=np.float64), np.ascontiguousarray(feq, dtype=np.float64)
        F = np.zeros(3) if force is None else np.ascontiguousarray(force, dtype=np.float64)
        uu = np.zeros(3) if u is None else np.ascontiguousarray(u, dtype=np.float64)
        return float(self.lib.zlp_smag_tau_sgs(dims, self._ptr(f), self._ptr(feq), tau0, dt, cs,
                                               1 if force is not None else 0, self._ptr(F), self._ptr(uu)))

    def tau(self, nu: float, level: int = 0) -> float:
        return float(self.lib.zlp_tau(nu, level))


def tgv_init(cfg: LevelConfig, u0: float, port: Port | None = None) -> np.ndarray:
    """Taylor-Green initial populations on the stored nodes (x = 2*pi*i/cells), feq from the oracle."""
    port = port or Port()
    cells = [v - 1 for v in cfg.n[: cfg.dims]]
    # coordinates modulo the period: the duplicated max plane starts identical to the min plane
    axes = [2.0 * np.pi * (np.arange(v) % c) / c for v, c in zip(cfg.n[: cfg.dims], cells)]
    if cfg.dims == 3:
        z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
        ux = u0 * np.sin(x) * np.cos(y) * np.cos(z)
        uy = -u0 * np.cos(x) * np.sin(y) * np.cos(z)
        uz = np.zeros_like(ux)
        p = cfg.rho0 * u0 * u0 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
        vel = np.stack([ux, uy, uz], -1)
    else:
        y, x = np.meshgrid(axes[1], axes[0], indexing="ij")
        ux = u0 * np.sin(x) * np.cos(y)
        uy = -u0 * np.cos(x) * np.sin(y)
        p = cfg.rho0 * u0 * u0 / 4.0 * (np.cos(2 * x) + np.cos(2 * y))
        vel = np.stack([ux, uy], -1)
    rho = cfg.rho0 + 3.0 * p
    f = np.empty(rho.shape + (cfg.q,))
    for idx in np.ndindex(rho.shape):
        f[idx] = port.feq(cfg.dims, float(rho[idx]), vel[idx])
    return f


def run_reference(cfg: LevelConfig, steps: int, workdir: str, init: str = "eq", u0: float = 0.05,
                  extra: list | None = None):
    """Run the reference harness; returns (records_before, records_after)."""
    workdir = os.path.abspath(workdir)
    os.makedirs(workdir, exist_ok=True)
    out0 = os.path.join(workdir, "before.bin")
    out1 = os.path.join(workdir, "after.bin")
    args = [REF_RUN] + cfg.harness_args() + [f"steps={steps}", f"init={init}", f"u0={u0!r}",
                                             f"out0={out0}", f"out={out1}"] + (extra or [])
    subprocess.run(args, check=True, cwd=workdir, stdout=subprocess.DEVNULL)
    return load_dump(out0)[2], load_dump(out1)[2]


# ---- Morton neighbour arithmetic (restates amr_project/grid/morton_aux.hpp:65-297) ----
def _axis_mask(dims: int, axis: int) -> int:
    nb = 64 // dims
    m = 0
    for i in range(nb):
        m |= 1 << (dims * i + axis)
    return m


def morton_neg(code: int, dims: int, axis: int) -> int:
    """FindXNeg/FindYNeg/FindZNeg: returns the input when the axis field is zero."""
    mk = _axis_mask(dims, axis)
    others = 0
    for a in range(dims):
        if a != axis:
            others |= _axis_mask(dims, a)
    v = code & mk
    if v == 0:
        return code
    return ((v - 1) & mk) | (code & others)


def morton_pos(code: int, dims: int, axis: int) -> int:
    """FindXPos/FindYPos/FindZPos: carry through the other axes' bits, wrap at 64 bits."""
    mk = _axis_mask(dims, axis)
    others = 0
    for a in range(dims):
        if a != axis:
            others |= _axis_mask(dims, a)
    t = ((code | (~mk & (2**64 - 1))) + 1) & (2**64 - 1)
    return (t & mk) | (code & others)


LATTICE_C = {
    2: [(0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, 1), (-1, -1), (1, -1)],
    3: [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (1, 1, 0), (-1, 1, 0),
        (1, -1, 0), (-1, -1, 0), (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1), (0, 1, 1), (0, -1, 1), (0, 1, -1),
        (0, -1, -1)],
}


def upstream_lookup(codes, dims: int) -> np.ndarray:
    """Position of node x - c_q in `codes` (or -1), by Morton steps and a dict lookup, the way the
    reference's stream finds its source nodes in the level's hash map."""
    codes = [int(c) for c in np.asarray(codes, dtype=np.uint64)]
    where = {c: i for i, c in enumerate(codes)}
    cs = LATTICE_C[dims]
    out = np.full((len(codes), len(cs)), -1, dtype=np.int64)
    for i, code in enumerate(codes):
        for q, c in enumerate(cs):
            u = code
            for a in range(dims):
                if c[a] > 0:
                    u = morton_neg(u, dims, a)
                elif c[a] < 0:
                    u = morton_pos(u, dims, a)
            out[i, q] = where.get(u, -1)
    return out


def load_levels(path: str):
    """Read a multi-level dump of ``ref_harness.cpp`` (``lout0=`` / ``lout=``).

    Returns (dims, q, levels) where each level is a dict with ``nodes`` (structured array of
    code, flag, rho, u[3], f[q], sorted by code) and ``layers`` {(kind, layer): codes}; kinds
    0/1 are the inner/outer coarse-to-fine layers of the level, 2/3 its inner/outer
    fine-to-coarse layers (grid/grid_info_interface.h:117-127)."""
    with open(path, "rb") as fh:
        raw = fh.read()
    dims, q, nlev = (int(v) for v in np.frombuffer(raw[:12], np.int32))
    off = 12
    rec = np.dtype([("code", "<u8"), ("flag", "<i4"), ("pad", "<i4"), ("rho", "<f8"), ("u", "<f8", (3,)),
                    ("f", "<f8", (q,))])
    levels = []
    for _ in range(nlev):
        n = int(np.frombuffer(raw[off:off + 8], np.int64)[0])
        off += 8
        nodes = np.frombuffer(raw[off:off + n * rec.itemsize], rec, count=n)
        off += n * rec.itemsize
        layers = {}
        while True:
            kind, layer = (int(v) for v in np.frombuffer(raw[off:off + 8], np.int32))
            off += 8
            if kind < 0:
                break
            c = int(np.frombuffer(raw[off:off + 8], np.int64)[0])
            off += 8
            codes = np.frombuffer(raw[off:off + 8 * c], np.uint64, count=c)
            off += 8 * c
            key = (kind, layer)
            layers[key] = np.union1d(layers[key], codes) if key in layers else codes.copy()
        levels.append({"nodes": nodes, "layers": layers})
    return dims, q, levels
