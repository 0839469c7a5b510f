"""Compact storage of a multi-level node topology: per level, the bounding box of its nodes and
bit masks (zlib-compressed) of the node set, the explosion targets (coarse-to-fine layers), the
coalescence targets and the coarse-to-fine ghost nodes excluded as explosion sources.  Refined
regions around a body are boxes with box-shaped holes and shell-shaped layers, so a few KB hold
grids of millions of nodes.

    python -m zllbm_b200.topology_pack IN.npz OUT.npz     # pack a topology archive

``IN.npz`` has the layout written by the host's grid builder (``codes<l>``, ``flags<l>``,
``c2f_fine<l>``, ``f2c_coarse<l>``, ``meta``); ``load`` returns that layout back, with
``flags<l>`` reduced to the ghost bit (4) that the flow drivers read.
"""
from __future__ import annotations

import json
import sys
import zlib

import numpy as np

SETS = ("codes", "c2f_fine", "f2c_coarse", "excluded")


def _decode(codes: np.ndarray, dims: int) -> np.ndarray:
    codes = np.asarray(codes, dtype=np.uint64)
    out = np.zeros((codes.size, dims), dtype=np.int64)
    for i in range(64 // dims):
        for a in range(dims):
            out[:, a] |= ((codes >> np.uint64(dims * i + a)) & np.uint64(1)).astype(np.int64) << i
    return out


def _encode(idx: np.ndarray, dims: int) -> np.ndarray:
    idx = np.asarray(idx, dtype=np.uint64)
    out = np.zeros(idx.shape[0], dtype=np.uint64)
    for i in range(64 // dims):
        for a in range(dims):
            out |= ((idx[:, a] >> np.uint64(i)) & np.uint64(1)) << np.uint64(dims * i + a)
    return out


def _mask(codes: np.ndarray, dims: int, lo: np.ndarray, shape: np.ndarray) -> bytes:
    m = np.zeros(int(np.prod(shape)), dtype=bool)
    if codes.size:
        idx = _decode(codes, dims) - lo
        if (idx < 0).any() or (idx >= shape).any():
            raise ValueError("code outside the level's bounding box")
        lin = idx[:, 0]
        stride = 1
        for a in range(1, dims):
            stride *= int(shape[a - 1])
            lin = lin + idx[:, a] * stride
        m[lin] = True
    return zlib.compress(np.packbits(m).tobytes(), 9)


def _unmask(blob: bytes, dims: int, lo: np.ndarray, shape: np.ndarray) -> np.ndarray:
    total = int(np.prod(shape))
    m = np.unpackbits(np.frombuffer(zlib.decompress(blob), dtype=np.uint8), count=total).astype(bool)
    lin = np.flatnonzero(m)
    idx = np.empty((lin.size, dims), dtype=np.int64)
    rest = lin
    for a in range(dims):
        idx[:, a] = rest % int(shape[a])
        rest = rest // int(shape[a])
    return np.sort(_encode(idx + lo, dims))


def pack(src: dict) -> dict:
    """Packed form of a topology archive (dict-like: codes<l>, flags<l>, c2f_fine<l>, f2c_coarse<l>, meta)."""
    meta = json.loads(str(src["meta"]))
    dims = int(meta["dims"])
    out = {"meta": json.dumps(meta)}
    lv = 0
    while f"codes{lv}" in src:
        codes = np.asarray(src[f"codes{lv}"], dtype=np.uint64)
        idx = _decode(codes, dims)
        lo, hi = idx.min(0), idx.max(0)
        shape = hi - lo + 1
        sets = {"codes": codes, "c2f_fine": src[f"c2f_fine{lv}"], "f2c_coarse": src[f"f2c_coarse{lv}"],
                "excluded": codes[(np.asarray(src[f"flags{lv}"]) & 4) != 0]}
        out[f"box{lv}"] = np.concatenate([lo, shape]).astype(np.int64)
        for name in SETS:
            out[f"{name}{lv}"] = np.frombuffer(_mask(np.asarray(sets[name], dtype=np.uint64), dims, lo, shape),
                                               dtype=np.uint8)
        lv += 1
    return out


def load(path: str) -> dict:
    """Unpacked topology in the builder's layout (flags reduced to the ghost bit 4)."""
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    dims = int(meta["dims"])
    out = {"meta": json.dumps(meta)}
    lv = 0
    while f"box{lv}" in z.files:
        box = z[f"box{lv}"]
        lo, shape = box[:dims], box[dims:]
        sets = {name: _unmask(z[f"{name}{lv}"].tobytes(), dims, lo, shape) for name in SETS}
        out[f"codes{lv}"] = sets["codes"]
        flags = np.zeros(sets["codes"].size, dtype=np.int32)
        flags[np.isin(sets["codes"], sets["excluded"])] = 4
        out[f"flags{lv}"] = flags
        out[f"c2f_fine{lv}"] = sets["c2f_fine"]
        out[f"f2c_coarse{lv}"] = sets["f2c_coarse"]
        lv += 1
    return out


def load_topology(path: str):
    """A topology archive in the builder's layout, packed (``box<l>`` entries) or not."""
    z = np.load(path)
    return load(path) if "box0" in z.files else z


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 2:
        raise SystemExit("usage: python -m zllbm_b200.topology_pack IN.npz OUT.npz")
    src = np.load(argv[0])
    np.savez_compressed(argv[1], **pack({k: src[k] for k in src.files}))


if __name__ == "__main__":
    main()
