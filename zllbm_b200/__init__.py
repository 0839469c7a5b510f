"""zllbm_b200 — B200-native lattice-Boltzmann time step over ZLLBM's Morton-coded grid.

The product is the CUDA library ``libzllbm_b200.so`` behind the C ABI declared in
``include/zllbm_b200.h``.  This module is a thin ctypes binding over that ABI for
Python callers (tests, benchmarks); it contains no numerics of its own and there
is no CPU fallback: if the library is missing or no GPU is present, calls fail.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libzllbm_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "zllbm_b200.h")

D2Q9, D3Q19 = 2, 3
SRT, MRT = 0, 1
BC_NONE, BC_BOUNCE_BACK, BC_PERIODIC, BC_NONEQ_EXTRAPOLATION, BC_CONVECTIVE_OUTFLOW = 0, 1, 2, 3, 4
STORAGE_F64, STORAGE_F32, STORAGE_F16, STORAGE_BF16 = 0, 1, 2, 3
STORAGE_NAMES = {"f64": STORAGE_F64, "f32": STORAGE_F32, "f16": STORAGE_F16, "bf16": STORAGE_BF16}
BLOCK_ROW = 1 << 20  # zl_set_block x: one warp per x-row (ZL_BLOCK_ROW)
ROUND_STOCHASTIC, ROUND_NEAREST = 0, 1  # zl_config.storage_rounding (stochastic is the default)
ABI_VERSION = 2
ERRORS = {-1: "EINVAL", -2: "ETOPOLOGY", -3: "EDEVICE", -4: "ETIMEOUT", -5: "ENAN", -6: "ESTATE",
          -7: "ETOOLARGE"}


class ZlError(RuntimeError):
    """A non-zero return from the C ABI (the reference logs these through LogManager::LogError)."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


class ZlConfig(ctypes.Structure):
    _fields_ = [
        ("lattice", ctypes.c_int),
        ("collision", ctypes.c_int),
        ("storage", ctypes.c_int),
        ("max_level", ctypes.c_int),
        ("viscosity", ctypes.c_double),
        ("rho0", ctypes.c_double),
        ("bc_kind", ctypes.c_int * 6),
        ("bc_velocity", (ctypes.c_double * 3) * 6),
        ("domain_min", ctypes.c_int32 * 3),
        ("domain_max", ctypes.c_int32 * 3),
        ("init_velocity", ctypes.c_double * 3),
        ("storage_scale", ctypes.c_double),
        ("forcing", ctypes.c_int),
        ("constant_force", ctypes.c_double * 3),
        ("les", ctypes.c_int),
        ("les_cs", ctypes.c_double),
        ("dx", ctypes.c_double),
        ("device", ctypes.c_int),
        ("storage_rounding", ctypes.c_int),
    ]


MLP_IN, MLP_HIDDEN, MLP_TRAINABLE = 24, 64, 5825
LES_OFF, LES_SMAGORINSKY, LES_LEARNED = 0, 1, 2


class ZlMlp(ctypes.Structure):
    """zl_mlp: the closure network's parameters (FP32), flat order w1 b1 w2 b2 w3 b3 mean inv_std."""
    _fields_ = [
        ("w1", ctypes.c_float * (MLP_HIDDEN * MLP_IN)),
        ("b1", ctypes.c_float * MLP_HIDDEN),
        ("w2", ctypes.c_float * (MLP_HIDDEN * MLP_HIDDEN)),
        ("b2", ctypes.c_float * MLP_HIDDEN),
        ("w3", ctypes.c_float * MLP_HIDDEN),
        ("b3", ctypes.c_float),
        ("in_mean", ctypes.c_float * MLP_IN),
        ("in_inv_std", ctypes.c_float * MLP_IN),
    ]

    @staticmethod
    def from_flat(v) -> "ZlMlp":
        v = np.ascontiguousarray(np.asarray(v, dtype=np.float32))
        assert v.size == ctypes.sizeof(ZlMlp) // 4
        m = ZlMlp()
        ctypes.memmove(ctypes.addressof(m), v.ctypes.data, v.nbytes)
        return m

    def flat(self) -> np.ndarray:
        out = np.empty(ctypes.sizeof(ZlMlp) // 4, dtype=np.float32)
        ctypes.memmove(out.ctypes.data, ctypes.addressof(self), out.nbytes)
        return out


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"zllbm_b200 CUDA library not built: {path} (run python -m zllbm_b200.build)")
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    i64 = ctypes.c_int64
    u64p = ctypes.POINTER(ctypes.c_uint64)
    dp = ctypes.POINTER(ctypes.c_double)
    sig = {
        "zl_abi_version": ([], ctypes.c_int),
        "zl_set_level_halo": ([P, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "zl_halo_bytes": ([P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "zl_halo_pack": ([P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
        "zl_halo_unpack": ([P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
        "zl_create": ([ctypes.POINTER(ZlConfig), ctypes.POINTER(P)], ctypes.c_int),
        "zl_destroy": ([P], ctypes.c_int),
        "zl_set_level_nodes": ([P, ctypes.c_int, u64p, i64], ctypes.c_int),
        "zl_set_populations": ([P, ctypes.c_int, u64p, dp, i64], ctypes.c_int),
        "zl_get_populations": ([P, ctypes.c_int, u64p, dp, i64], ctypes.c_int),
        "zl_get_macros": ([P, ctypes.c_int, u64p, dp, dp, i64], ctypes.c_int),
        "zl_step_level": ([P, ctypes.c_int], ctypes.c_int),
        "zl_step_level_planes": ([P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "zl_advance": ([P, ctypes.c_int], ctypes.c_int),
        "zl_set_level_interface": ([P, ctypes.c_int, u64p, i64, u64p, i64, u64p, i64], ctypes.c_int),
        "zl_transfer_levels": ([P, ctypes.c_int], ctypes.c_int),
        "zl_set_graph": ([P, ctypes.c_int], ctypes.c_int),
        "zl_set_batching": ([P, ctypes.c_int], ctypes.c_int),
        "zl_set_level_streams": ([P, ctypes.c_int], ctypes.c_int),
        "zl_set_block": ([P, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "zl_write_checkpoint_nodes": ([P, ctypes.c_char_p, ctypes.POINTER(u64p),
                                       ctypes.POINTER(ctypes.POINTER(ctypes.c_int32)), ctypes.POINTER(i64)],
                                      ctypes.c_int),
        "zl_read_checkpoint_nodes": ([P, ctypes.c_char_p], ctypes.c_int),
        "zl_write_vtu": ([P, ctypes.c_char_p, ctypes.c_int, dp, dp, ctypes.c_uint32, ctypes.POINTER(u64p),
                          ctypes.POINTER(ctypes.POINTER(ctypes.c_int32)), ctypes.POINTER(i64)], ctypes.c_int),
        "zl_set_temporal_interpolation": ([P, ctypes.c_int], ctypes.c_int),
        "zl_interpolate_interface": ([P, ctypes.c_int], ctypes.c_int),
        "zl_autotune": ([P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
        "zl_conservation": ([P, ctypes.c_int, dp], ctypes.c_int),
        "zl_synchronize": ([P], ctypes.c_int),
        "zl_get_stream": ([P, ctypes.POINTER(P)], ctypes.c_int),
        "zl_set_stream": ([P, P], ctypes.c_int),
        "zl_last_error": ([P, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
        "zl_level_info": ([P, ctypes.c_int, ctypes.POINTER(i64), ctypes.POINTER(ctypes.c_int32),
                           ctypes.POINTER(i64)], ctypes.c_int),
        "zl_morton_neighbors": ([ctypes.c_int, u64p, i64, u64p], ctypes.c_int),
        "zl_upstream_index": ([ctypes.c_int, u64p, i64, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "zl_mrt_matrix": ([ctypes.c_int, ctypes.c_double, dp], ctypes.c_int),
        "zl_moments_noalloc": ([ctypes.c_int, P, i64, P, P], ctypes.c_int),
        "zl_ib_set_vertices": ([P, ctypes.c_int, i64, dp, dp, dp], ctypes.c_int),
        "zl_ib_get_forces": ([P, ctypes.c_int, dp, dp], ctypes.c_int),
        "zl_ib_set_delta": ([P, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "zl_set_level_box": ([P, ctypes.c_int, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)],
                             ctypes.c_int),
        "zl_set_equilibrium_dense": ([P, ctypes.c_int, P, P], ctypes.c_int),
        "zl_get_macros_dense": ([P, ctypes.c_int, P, P], ctypes.c_int),
        "zl_set_closure": ([P, ctypes.POINTER(ZlMlp)], ctypes.c_int),
        "zl_set_closure_interval": ([P, ctypes.c_int], ctypes.c_int),
        "zl_closure_features": ([P, ctypes.c_int, P], ctypes.c_int),
        "zl_filter_level": ([P, ctypes.c_int, ctypes.c_int, P], ctypes.c_int),
        "zl_closure_pairs": ([ctypes.POINTER(ctypes.c_int32), P, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                              P, P, P, P], ctypes.c_int),
        "zl_mlp_forward": ([ctypes.POINTER(ZlMlp), P, i64, P, P], ctypes.c_int),
        "zl_trainer_create": ([ctypes.POINTER(ZlMlp), ctypes.c_int, ctypes.POINTER(P)], ctypes.c_int),
        "zl_trainer_step": ([P, P, P, i64, ctypes.c_float], ctypes.c_int),
        "zl_trainer_set_stream": ([P, P], ctypes.c_int),
        "zl_trainer_loss": ([P, dp], ctypes.c_int),
        "zl_trainer_gradients": ([P, ctypes.POINTER(ZlMlp)], ctypes.c_int),
        "zl_trainer_weights": ([P, ctypes.POINTER(ZlMlp)], ctypes.c_int),
        "zl_trainer_destroy": ([P], None),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def header_symbols(path: str = HEADER) -> list[str]:
    """Function names declared in include/zllbm_b200.h."""
    import re

    text = open(path).read()
    return sorted(set(re.findall(r"^\s*(?:int|void)\s+(zl_\w+)\s*\(", text, flags=re.M)))


def _u64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _p(a: np.ndarray, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


@dataclass
class SolverConfig:
    """Mirror of the settings a reference application makes on SolverLbmInterface / GridManager."""

    lattice: int = D3Q19
    collision: int = SRT
    storage: int = STORAGE_F64
    max_level: int = 0
    viscosity: float = 0.1
    rho0: float = 1.0
    bc_kind: tuple = (0, 0, 0, 0, 0, 0)
    bc_velocity: tuple = ((0.0, 0.0, 0.0),) * 6
    domain_min: tuple = (1, 1, 1)
    domain_max: tuple = (2, 2, 2)
    init_velocity: tuple = (0.0, 0.0, 0.0)
    storage_scale: float = 0.0
    forcing: int = 0
    constant_force: tuple = (0.0, 0.0, 0.0)
    les: int = 0
    les_cs: float = 0.0
    dx: float = 0.0
    device: int = 0
    storage_rounding: int = 0  # ROUND_STOCHASTIC (default) or ROUND_NEAREST (FP16 / BF16 storage)
    extra: dict = field(default_factory=dict)

    @property
    def dims(self) -> int:
        return 2 if self.lattice == D2Q9 else 3

    @property
    def q(self) -> int:
        return 9 if self.lattice == D2Q9 else 19

    def to_c(self) -> ZlConfig:
        c = ZlConfig()
        c.lattice, c.collision, c.storage, c.max_level = self.lattice, self.collision, self.storage, self.max_level
        c.viscosity, c.rho0 = self.viscosity, self.rho0
        for f in range(6):
            c.bc_kind[f] = int(self.bc_kind[f])
            for a in range(3):
                c.bc_velocity[f][a] = float(self.bc_velocity[f][a]) if a < len(self.bc_velocity[f]) else 0.0
        for a in range(3):
            c.domain_min[a] = int(self.domain_min[a]) if a < len(self.domain_min) else 0
            c.domain_max[a] = int(self.domain_max[a]) if a < len(self.domain_max) else 0
            c.init_velocity[a] = float(self.init_velocity[a]) if a < len(self.init_velocity) else 0.0
        c.storage_scale = self.storage_scale
        c.forcing = self.forcing
        for a in range(3):
            c.constant_force[a] = float(self.constant_force[a]) if a < len(self.constant_force) else 0.0
        c.les = self.les
        c.les_cs = self.les_cs
        c.dx = self.dx
        c.device = self.device
        c.storage_rounding = self.storage_rounding
        return c


class Context:
    """One device context (zl_create / zl_destroy)."""

    def __init__(self, config: SolverConfig):
        self.lib = load_library()
        self.config = config
        h = ctypes.c_void_p()
        self._cfg = config.to_c()
        rc = self.lib.zl_create(ctypes.byref(self._cfg), ctypes.byref(h))
        if rc != 0:
            raise ZlError(rc, "zl_create failed")
        self.handle = h

    def _check(self, rc: int):
        if rc != 0:
            buf = ctypes.create_string_buffer(512)
            self.lib.zl_last_error(self.handle, buf, 512)
            raise ZlError(rc, buf.value.decode(errors="replace"))

    def close(self):
        if getattr(self, "handle", None):
            self.lib.zl_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_level_nodes(self, level: int, codes):
        c = _u64(codes)
        self._check(self.lib.zl_set_level_nodes(self.handle, level, _p(c, ctypes.c_uint64), c.size))

    def _node_list(self, codes, n: int | None = None):
        """(pointer, count) of an exchange's node list; codes None: the level's own list in the
        order of set_level_nodes (count n), kept on the device and not uploaded again."""
        if codes is None:
            if n is None:
                raise ValueError("without codes the node count is needed")
            return None, int(n), None
        c = _u64(codes)
        return _p(c, ctypes.c_uint64), c.size, c

    def set_populations(self, level: int, codes, f):
        ff = _f64(f)
        ptr, n, keep = self._node_list(codes, ff.size // self.config.q)
        assert ff.size == n * self.config.q
        self._check(self.lib.zl_set_populations(self.handle, level, ptr, _p(ff, ctypes.c_double), n))

    def get_populations(self, level: int, codes, n: int | None = None) -> np.ndarray:
        ptr, n, keep = self._node_list(codes, n)
        out = np.empty((n, self.config.q))
        self._check(self.lib.zl_get_populations(self.handle, level, ptr, _p(out, ctypes.c_double), n))
        return out

    def get_macros(self, level: int, codes, n: int | None = None):
        ptr, n, keep = self._node_list(codes, n)
        rho = np.empty(n)
        u = np.empty((n, self.config.dims))
        self._check(self.lib.zl_get_macros(self.handle, level, ptr, _p(rho, ctypes.c_double),
                                           _p(u, ctypes.c_double), n))
        return rho, u

    def set_level_interface(self, level: int, c2f_fine, f2c_coarse, coarse_excluded):
        a, b, c = _u64(c2f_fine), _u64(f2c_coarse), _u64(coarse_excluded)
        self._check(self.lib.zl_set_level_interface(self.handle, level, _p(a, ctypes.c_uint64), a.size,
                                                    _p(b, ctypes.c_uint64), b.size, _p(c, ctypes.c_uint64), c.size))

    def transfer_levels(self, fine_level: int):
        self._check(self.lib.zl_transfer_levels(self.handle, fine_level))

    def set_temporal_interpolation(self, enabled: bool):
        self._check(self.lib.zl_set_temporal_interpolation(self.handle, 1 if enabled else 0))

    def interpolate_interface(self, fine_level: int):
        self._check(self.lib.zl_interpolate_interface(self.handle, fine_level))

    def set_level_halo(self, level: int, faces: int):
        """Faces (bit f = face slot f) whose ghost cells hold a neighbouring slab's slots."""
        self._check(self.lib.zl_set_level_halo(self.handle, level, faces))

    def halo_bytes(self, level: int, face: int) -> int:
        out = ctypes.c_int64()
        self._check(self.lib.zl_halo_bytes(self.handle, level, face, ctypes.byref(out)))
        return out.value

    def halo_pack(self, level: int, face: int, stage: int, buf_ptr: int):
        self._check(self.lib.zl_halo_pack(self.handle, level, face, stage, ctypes.c_void_p(buf_ptr)))

    def halo_unpack(self, level: int, face: int, stage: int, buf_ptr: int):
        self._check(self.lib.zl_halo_unpack(self.handle, level, face, stage, ctypes.c_void_p(buf_ptr)))

    def set_block(self, level: int, x: int, y: int = 1):
        """Step-kernel block shape; negative x: two nodes per thread (packed FP32 pairs);
        x = BLOCK_ROW: one warp per x-row, y rows per block."""
        self._check(self.lib.zl_set_block(self.handle, level, x, y))

    def write_checkpoint_nodes(self, path: str, codes: list, flags: list):
        """The reference's grid_nodes checkpoint file from the device state; codes[l], flags[l]
        per level 0 .. max_level."""
        levels = len(codes)
        cs = [_u64(c) for c in codes]
        fs = [np.ascontiguousarray(np.asarray(f, dtype=np.int32)) for f in flags]
        cp = (ctypes.POINTER(ctypes.c_uint64) * levels)(*[_p(c, ctypes.c_uint64) for c in cs])
        fp = (ctypes.POINTER(ctypes.c_int32) * levels)(*[_p(f, ctypes.c_int32) for f in fs])
        n = (ctypes.c_int64 * levels)(*[c.size for c in cs])
        self._check(self.lib.zl_write_checkpoint_nodes(self.handle, path.encode(), cp, fp, n))

    def write_vtu(self, prefix: str, codes: list, flags: list, binary: bool = True, space=(1.0, 1.0, 1.0),
                  origin=(-1.0, -1.0, -1.0), ghost_mask: int = 0x3E):
        """The reference's VTK XML field output (<prefix>_data/rank_0_grid_level_<l>.vtu and
        rank_0_.pvtu); codes[l], flags[l]: level l's points in output order with their flag_status.
        origin defaults to -spacing * 1, the reference's minimum background node index."""
        levels = len(codes)
        cs = [_u64(c) for c in codes]
        fs = [np.ascontiguousarray(np.asarray(f, dtype=np.int32)) for f in flags]
        cp = (ctypes.POINTER(ctypes.c_uint64) * levels)(*[_p(c, ctypes.c_uint64) for c in cs])
        fp = (ctypes.POINTER(ctypes.c_int32) * levels)(*[_p(f, ctypes.c_int32) for f in fs])
        n = (ctypes.c_int64 * levels)(*[c.size for c in cs])
        sp = (ctypes.c_double * 3)(*space)
        og = (ctypes.c_double * 3)(*origin)
        self._check(self.lib.zl_write_vtu(self.handle, prefix.encode(), 1 if binary else 0, sp, og,
                                          ctypes.c_uint32(ghost_mask), cp, fp, n))

    def read_checkpoint_nodes(self, path: str):
        self._check(self.lib.zl_read_checkpoint_nodes(self.handle, path.encode()))

    def set_batching(self, enabled: bool):
        self._check(self.lib.zl_set_batching(self.handle, 1 if enabled else 0))

    def set_level_streams(self, enabled: bool):
        self._check(self.lib.zl_set_level_streams(self.handle, 1 if enabled else 0))

    def set_graph(self, enabled: bool):
        self._check(self.lib.zl_set_graph(self.handle, 1 if enabled else 0))

    def autotune(self, level: int = 0, trials: int = 8):
        out = (ctypes.c_int32 * 2)()
        self._check(self.lib.zl_autotune(self.handle, level, trials, out))
        return tuple(out)

    def step_level(self, level: int = 0):
        self._check(self.lib.zl_step_level(self.handle, level))

    def step_level_planes(self, level: int, first: int, count: int, finish: bool):
        """Planes [first, first + count) of the level's last axis; finish completes the step."""
        self._check(self.lib.zl_step_level_planes(self.handle, level, first, count, 1 if finish else 0))

    def advance(self, steps: int):
        self._check(self.lib.zl_advance(self.handle, steps))

    def conservation(self, level: int = 0) -> np.ndarray:
        out = np.zeros(4)
        self._check(self.lib.zl_conservation(self.handle, level, _p(out, ctypes.c_double)))
        return out[: self.config.dims + 1]

    def synchronize(self):
        self._check(self.lib.zl_synchronize(self.handle))

    def ib_set_vertices(self, level: int, coordinates, velocity, area):
        c, v, a = _f64(coordinates).reshape(-1, 3), _f64(velocity).reshape(-1, 3), _f64(area).ravel()
        c, v = np.ascontiguousarray(c), np.ascontiguousarray(v)
        self._check(self.lib.zl_ib_set_vertices(self.handle, level, a.size, _p(c, ctypes.c_double),
                                                _p(v, ctypes.c_double), _p(a, ctypes.c_double)))
        self._nv = {**getattr(self, "_nv", {}), level: a.size}

    def ib_set_delta(self, level: int, width: int):
        """Stencil width of the delta kernel: 4 (reference) or 3 (Roma, Peskin and Berger)."""
        self._check(self.lib.zl_ib_set_delta(self.handle, level, width))

    def ib_get_forces(self, level: int):
        n = self._nv[level]
        forces = np.empty((n, 3))
        total = np.empty(3)
        self._check(self.lib.zl_ib_get_forces(self.handle, level, _p(forces, ctypes.c_double),
                                              _p(total, ctypes.c_double)))
        return forces, total

    def stream(self) -> int:
        """The cudaStream_t the context issues work on (as an integer handle)."""
        h = ctypes.c_void_p()
        self._check(self.lib.zl_get_stream(self.handle, ctypes.byref(h)))
        return h.value or 0

    def set_stream(self, stream: int | None):
        self._check(self.lib.zl_set_stream(self.handle, ctypes.c_void_p(stream) if stream else None))

    # full-box levels and device I/O (device pointers as integers, e.g. torch tensor data_ptr())
    def set_level_box(self, level: int, lo, n):
        lo_c = (ctypes.c_int32 * 3)(*[int(v) for v in lo])
        n_c = (ctypes.c_int32 * 3)(*[int(v) for v in n])
        self._check(self.lib.zl_set_level_box(self.handle, level, lo_c, n_c))

    def set_equilibrium_dense(self, level: int, rho_ptr: int, u_ptr: int):
        self._check(self.lib.zl_set_equilibrium_dense(self.handle, level, ctypes.c_void_p(rho_ptr),
                                                      ctypes.c_void_p(u_ptr)))

    def get_macros_dense(self, level: int, rho_ptr: int, u_ptr: int):
        self._check(self.lib.zl_get_macros_dense(self.handle, level, ctypes.c_void_p(rho_ptr), ctypes.c_void_p(u_ptr)))

    def closure_features(self, level: int, x_ptr: int):
        self._check(self.lib.zl_closure_features(self.handle, level, ctypes.c_void_p(x_ptr)))

    def filter_level(self, level: int, factor: int, out_ptr: int):
        self._check(self.lib.zl_filter_level(self.handle, level, factor, ctypes.c_void_p(out_ptr)))

    def set_closure_interval(self, every: int):
        self._check(self.lib.zl_set_closure_interval(self.handle, every))

    def set_closure(self, net: "ZlMlp | None"):
        self._check(self.lib.zl_set_closure(self.handle, ctypes.byref(net) if net is not None else None))

    def level_info(self, level: int = 0):
        n = ctypes.c_int64()
        ext = (ctypes.c_int32 * 3)()
        pb = ctypes.c_int64()
        self._check(self.lib.zl_level_info(self.handle, level, ctypes.byref(n), ext, ctypes.byref(pb)))
        return n.value, tuple(ext), pb.value


def morton_neighbors(dims: int, codes) -> np.ndarray:
    lib = load_library()
    c = _u64(codes)
    out = np.empty((c.size, 2 * dims), dtype=np.uint64)
    rc = lib.zl_morton_neighbors(dims, _p(c, ctypes.c_uint64), c.size, _p(out, ctypes.c_uint64))
    if rc:
        raise ZlError(rc, "zl_morton_neighbors")
    return out


def upstream_index(lattice: int, codes) -> np.ndarray:
    lib = load_library()
    c = _u64(codes)
    q = 9 if lattice == D2Q9 else 19
    out = np.empty((c.size, q), dtype=np.int64)
    rc = lib.zl_upstream_index(lattice, _p(c, ctypes.c_uint64), c.size, _p(out, ctypes.c_int64))
    if rc:
        raise ZlError(rc, "zl_upstream_index")
    return out


def mrt_matrix(lattice: int, tau: float) -> np.ndarray:
    lib = load_library()
    q = 9 if lattice == D2Q9 else 19
    out = np.empty(q * q)
    rc = lib.zl_mrt_matrix(lattice, tau, _p(out, ctypes.c_double))
    if rc:
        raise ZlError(rc, "zl_mrt_matrix")
    return out.reshape(q, q)


def box_codes(dims: int, lo, hi) -> np.ndarray:
    """Morton codes of every node with lo <= index <= hi per axis, x fastest (host helper)."""
    axes = [np.arange(lo[a], hi[a] + 1, dtype=np.uint64) for a in range(dims)]
    grids = np.meshgrid(*reversed(axes), indexing="ij")
    idx = np.stack([g.ravel() for g in reversed(grids)], axis=1)
    out = np.zeros(idx.shape[0], dtype=np.uint64)
    for i in range(64 // dims):
        for a in range(dims):
            out |= ((idx[:, a] >> np.uint64(i)) & np.uint64(1)) << np.uint64(dims * i + a)
    return out


def closure_pairs(nc, filtered_ptr: int, tau_fine: float, tau_coarse: float, factor: int, x_ptr: int, y_ptr: int,
                  scratch_ptr: int, stream: int = 0):
    lib = load_library()
    n3 = (ctypes.c_int32 * 3)(*[int(v) for v in nc])
    rc = lib.zl_closure_pairs(n3, ctypes.c_void_p(filtered_ptr), tau_fine, tau_coarse, factor, ctypes.c_void_p(x_ptr),
                              ctypes.c_void_p(y_ptr), ctypes.c_void_p(scratch_ptr), ctypes.c_void_p(stream or None))
    if rc:
        raise ZlError(rc, "zl_closure_pairs")


def mlp_forward(net: ZlMlp, x_ptr: int, n: int, y_ptr: int, stream: int = 0):
    lib = load_library()
    rc = lib.zl_mlp_forward(ctypes.byref(net), ctypes.c_void_p(x_ptr), n, ctypes.c_void_p(y_ptr),
                            ctypes.c_void_p(stream or None))
    if rc:
        raise ZlError(rc, "zl_mlp_forward")


class Trainer:
    """zl_trainer: tensor-core training of the closure network (device arrays as integer pointers)."""

    def __init__(self, init: ZlMlp, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.zl_trainer_create(ctypes.byref(init), device, ctypes.byref(h))
        if rc:
            raise ZlError(rc, "zl_trainer_create")
        self.handle = h

    def _check(self, rc, what):
        if rc:
            raise ZlError(rc, what)

    def set_stream(self, stream: int | None):
        self._check(self.lib.zl_trainer_set_stream(self.handle, ctypes.c_void_p(stream) if stream else None),
                    "zl_trainer_set_stream")

    def step(self, x_ptr: int, y_ptr: int, n: int, lr: float):
        self._check(self.lib.zl_trainer_step(self.handle, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr), n, lr),
                    "zl_trainer_step")

    def loss(self) -> float:
        v = ctypes.c_double()
        self._check(self.lib.zl_trainer_loss(self.handle, ctypes.byref(v)), "zl_trainer_loss")
        return v.value

    def gradients(self) -> ZlMlp:
        g = ZlMlp()
        self._check(self.lib.zl_trainer_gradients(self.handle, ctypes.byref(g)), "zl_trainer_gradients")
        return g

    def weights(self) -> ZlMlp:
        w = ZlMlp()
        self._check(self.lib.zl_trainer_weights(self.handle, ctypes.byref(w)), "zl_trainer_weights")
        return w

    def close(self):
        if getattr(self, "handle", None):
            self.lib.zl_trainer_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
