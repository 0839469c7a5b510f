"""ORACLE — test infrastructure only.

Restatement of the node records of the reference's checkpoint file `grid_nodes`
(MpiManager::WriteCheckPointGridNodes, amr_project/mpi/mpi_checkpoint.cpp:272-380, node data
GridNodeLbm::CopyANodeToBufferForCheckpoint, lbm_project/lbm_interface.h:57-78):

    uint32 node count, int32 node data size,
    per node: uint64 code, int32 level, int32 flag_status_, double f_[q], double force_[n_forces]

Nodes are grouped by background cell (code >> dims * level, SFBitsetToNLowerLevel) in ascending
order of that cell's code (the std::map of ComputeComputationalLoadOnEachRank,
mpi_checkpoint.cpp:39-104); inside a cell, levels ascend and each level's nodes follow
SFBitsetHigherLevelInACell (sfbitset_aux.cpp:140-156, :1958-1985): x fastest, then y, then z.
"""
from __future__ import annotations

import numpy as np

from oracle.port import morton_decode


def record_dtype(q: int, n_forces: int) -> np.dtype:
    fields = [("code", "<u8"), ("level", "<i4"), ("flag", "<i4"), ("f", "<f8", (q,))]
    if n_forces:
        fields.append(("force", "<f8", (n_forces,)))
    return np.dtype(fields)


def order(dims: int, level_codes) -> list:
    """(level, index) of every node in the file's order."""
    keys = []
    for lv, codes in enumerate(level_codes):
        codes = np.asarray(codes, dtype=np.uint64)
        if codes.size == 0:
            continue
        bg = codes >> np.uint64(dims * lv)
        idx = morton_decode(codes, dims)
        side = 1 << lv
        local = np.zeros(codes.size, dtype=np.int64)
        for a in reversed(range(dims)):
            local = local * side + (idx[:, a] & (side - 1))
        for i in range(codes.size):
            keys.append((int(bg[i]), lv, int(local[i]), i))
    keys.sort()
    return [(lv, i) for _, lv, _, i in keys]


def grid_nodes(dims: int, levels, n_forces: int = 0) -> bytes:
    """levels: list of dicts with codes, flags, f (and force when n_forces) per level."""
    q = levels[0]["f"].shape[1]
    dt = record_dtype(q, n_forces)
    seq = order(dims, [lv["codes"] for lv in levels])
    rec = np.zeros(len(seq), dtype=dt)
    for k, (lv, i) in enumerate(seq):
        L = levels[lv]
        rec[k]["code"] = L["codes"][i]
        rec[k]["level"] = lv
        rec[k]["flag"] = L["flags"][i]
        rec[k]["f"] = L["f"][i]
        if n_forces:
            rec[k]["force"] = L["force"][i] if "force" in L else 0.0
    head = np.array([len(seq)], np.uint32).tobytes() + np.array([dt.itemsize - 12], np.int32).tobytes()
    return head + rec.tobytes()


def parse(raw: bytes, q: int):
    n = int(np.frombuffer(raw[:4], np.uint32)[0])
    size = int(np.frombuffer(raw[4:8], np.int32)[0])
    n_forces = (size - 4 - 8 * q) // 8
    return np.frombuffer(raw[8:], record_dtype(q, n_forces), count=n), n_forces
