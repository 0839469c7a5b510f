"""CPU restatement of the reference's VTK XML field output (test infrastructure only).

Follows amr_project/io/vtk_writer_manager.cpp with the default ghost-cell option
kPartitionMultiBlock (WriteVtuAll, :103-190): one ``rank_0_grid_level_<l>.vtu`` per level in
``<prefix>_data/`` and ``rank_0_.pvtu`` listing them.  Per level the points are written in a given
node order (the reference's hash-map order); per point flag_status (UInt16), vtkGhostType (UInt8,
1 where flag_status & overlap flags), the LBM output variables in std::set order "rho", "velocity"
(lbm_project/lbm_grid_interface.cpp:614-707, Float32), the coordinates (Float32 x 3, :1156-1176 of
the writer: background origin plus the level spacing times each set Morton bit) and VTK_PIXEL /
VTK_VOXEL cells for every point that is the lower corner of a cell whose corners all exist
(SFBitsetBelongToOneCell, amr_project/grid/sfbitset_aux.h:738-830: corner order (0,0,0), (+x),
(+y), (+x,+y), (+z), (+x,+z), (+y,+z), (+x,+y,+z)).  Binary arrays are base64 text of a UInt32
byte count followed by the data (Base64Utility::Encode, :29-77); ASCII arrays use the printf
formats of IoManager::SetupOutputFormat (io_manager.cpp:20-80).
"""
from __future__ import annotations

import base64

import numpy as np

from oracle.port import morton_decode

GHOST_FLAGS = (1 << 1) | (1 << 2) | (1 << 5) | (1 << 3) | (1 << 4)  # C2F0 | C2FGhost | MpiOuter | F2C0 | F2CGhost

C9 = np.array([(0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, 1), (-1, -1), (1, -1)], dtype=np.float64)


def output_macros(f: np.ndarray, dims: int, force=None, dt: float = 1.0):
    """Density and velocity of the "velocity" output variable: CalMacro{2D,3D}Compressible, or the
    forced form (lbm_project/lbm_solver_interface.cpp:477-592) when the solver has forces:
    rho = f0 + sum_{q>=1} f_q, u = (sum_q c_q f_q [+ 0.5 F dt]) / rho, in index order."""
    from oracle.closure import C19
    c = C9 if dims == 2 else C19.astype(np.float64)
    f = np.asarray(f, dtype=np.float64)
    rho = f[:, 0].copy()
    u = np.zeros((f.shape[0], dims))
    for q in range(1, f.shape[1]):
        rho = rho + f[:, q]
        for a in range(dims):
            u[:, a] = u[:, a] + c[q, a] * f[:, q]
    if force is not None:
        for a in range(dims):
            u[:, a] = u[:, a] + 0.5 * float(force[a]) * dt
    return rho, u / rho[:, None]


def b64(payload: bytes) -> bytes:
    return base64.b64encode(len(payload).to_bytes(4, "little") + payload)


def coordinates(codes: np.ndarray, dims: int, level: int, space, origin) -> np.ndarray:
    """SFBitsetComputeCoordinate (amr_project/grid/morton_aux.cpp:86-101, :310-333): origin plus
    spacing * 2^i for every set bit i of each axis, bits in ascending order."""
    codes = np.asarray(codes, dtype=np.uint64)
    out = np.zeros((codes.size, 3))
    for a in range(dims):
        gs = space[a] / float(1 << level)
        c = np.full(codes.size, float(origin[a]))
        for i in range(64 // dims):
            bit = (codes >> np.uint64(dims * i + a)) & np.uint64(1)
            c = np.where(bit == 1, c + gs * float(1 << i), c)
        out[:, a] = c
    return out


def cells(codes: np.ndarray, dims: int) -> np.ndarray:
    """Point indices of every cell, in point order of the cell's lower corner."""
    idx = morton_decode(np.asarray(codes, dtype=np.uint64), dims).astype(np.int64)
    where = {tuple(r): i for i, r in enumerate(idx)}
    corners = [(0, 0), (1, 0), (0, 1), (1, 1)] if dims == 2 else \
        [(0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0), (0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 1)]
    out = []
    for r in idx:
        pts = [where.get(tuple(r + np.array(c))) for c in corners]
        if all(p is not None for p in pts):
            out.append(pts)
    return np.array(out, dtype=np.uint64).reshape(-1, len(corners))


def _ascii_lines(fmt: str, rows) -> bytes:
    return b"".join((fmt % r).encode() for r in rows)


def level_vtu(binary: bool, dims: int, flags, rho, vel, coords, conn, ghost_flags: int = GHOST_FLAGS) -> bytes:
    """One level's .vtu (WriteVtuGrid + WriteGridPieces)."""
    fmt = "binary" if binary else "ascii"
    flags = np.asarray(flags, dtype=np.int64)
    n, nc = flags.size, conn.shape[0]
    corners = 4 if dims == 2 else 8
    ghost = ((flags & ghost_flags) != 0).astype(np.uint8)
    out = [b'<?xml version="1.0"?>\n',
           b'<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">\n',
           b" <UnstructuredGrid>\n",
           f'  <Piece NumberOfPoints="{n}" NumberOfCells="{nc}">\n'.encode(),
           b"    <PointData>\n",
           f'      <DataArray NumberOfComponents="1" type="UInt16" Name="flag_status" format="{fmt}">\n'.encode()]
    if binary:
        out.append(b64(flags.astype(np.uint16).tobytes()) + b"\n")
    else:
        out.append(_ascii_lines("       %d\n", (int(v) & 0xFFFF for v in flags)))
    out.append(b"      </DataArray>\n")
    out.append(f'      <DataArray type="UInt8" Name="vtkGhostType" format="{fmt}">\n'.encode())
    out.append(b64(ghost.tobytes()) + b"\n" if binary else _ascii_lines("   %d\n", (int(v) for v in ghost)))
    out.append(b"      </DataArray>\n")
    for name, arr, comps in (("rho", np.asarray(rho, dtype=np.float64).reshape(n, 1), 1),
                             ("velocity", np.asarray(vel, dtype=np.float64).reshape(n, dims), dims)):
        out.append(f'      <DataArray NumberOfComponents="{comps}" type="Float32" Name="{name}" '
                   f'format="{fmt}">\n'.encode())
        if binary:
            out.append(b64(arr.astype(np.float32).tobytes()) + b"\n")
        else:
            out.append(b"".join(("".join("  " + "     %f" % v for v in row) + "\n").encode() for row in arr))
        out.append(b"      </DataArray>\n")
    out.append(b"    </PointData>\n")
    out.append(b"   <Points>\n")
    out.append(f'    <DataArray type="Float32" NumberOfComponents="3" format="{fmt}">\n'.encode())
    out.append(b64(coords.astype(np.float32).tobytes()) + b"\n" if binary
               else _ascii_lines("   %f %f %f\n", (tuple(r) for r in coords)))
    out.append(b"    </DataArray>\n")
    out.append(b"   </Points>\n")
    out.append(b"   <Cells>\n")
    out.append(f'    <DataArray type="UInt64" Name="connectivity" format="{fmt}">\n'.encode())
    out.append(b64(conn.astype(np.uint64).tobytes()) + b"\n" if binary
               else b"".join(("  " + "".join(" %d" % int(v) for v in row) + "\n").encode() for row in conn))
    out.append(b"    </DataArray>\n")
    out.append(f'    <DataArray type="UInt64" Name="offsets" format="{fmt}">\n'.encode())
    offs = (np.arange(1, nc + 1, dtype=np.uint64) * np.uint64(corners))
    out.append(b64(offs.tobytes()) + b"\n" if binary else _ascii_lines("   %d\n", (int(v) for v in offs)))
    out.append(b"    </DataArray>\n")
    out.append(f'    <DataArray type="UInt8" Name="types" format="{fmt}">\n'.encode())
    types = np.full(nc, 8 if dims == 2 else 11, dtype=np.uint8)
    out.append(b64(types.tobytes()) + b"\n" if binary else _ascii_lines("   %d\n", (int(v) for v in types)))
    out.append(b"    </DataArray>\n")
    out.append(b"   </Cells>\n")
    out.append(b"  </Piece>\n")
    out.append(b" </UnstructuredGrid>\n")
    out.append(b"</VTKFile>")
    return b"".join(out)


def pvtu(binary: bool, dims: int, levels: int) -> bytes:
    """rank_0_.pvtu (WritePvtu, vtk_writer_manager.cpp:296-372)."""
    fmt = "binary" if binary else "ascii"
    out = [b'<?xml version="1.0"?>\n',
           b'<VTKFile type="PUnstructuredGrid" version="0.1" byte_order="LittleEndian">\n',
           b" <PUnstructuredGrid>\n",
           b"    <PPointData>\n",
           f'      <PDataArray NumberOfComponents="1" type="UInt16" Name="flag_status" format="{fmt}">\n'.encode(),
           b"      </PDataArray>\n",
           f'      <PDataArray NumberOfComponents="1" type="Float32" Name="rho" format="{fmt}">\n'.encode(),
           b"      </PDataArray>\n",
           f'      <PDataArray NumberOfComponents="{dims}" type="Float32" Name="velocity" format="{fmt}">\n'.encode(),
           b"      </PDataArray>\n",
           f'      <PDataArray type="UInt8" Name="vtkGhostType" format="{fmt}">\n'.encode(),
           b"      </PDataArray>\n",
           b"    </PPointData>\n",
           b"   <PPoints>\n",
           f'    <PDataArray type="Float32" NumberOfComponents="3" format="{fmt}">\n'.encode(),
           b"    </PDataArray>\n",
           b"   </PPoints>\n",
           b"   <PCells>\n",
           f'    <PDataArray type="UInt64" Name="connectivity" format="{fmt}">\n'.encode(),
           b"    </PDataArray>\n",
           f'    <PDataArray type="UInt64" Name="offsets" format="{fmt}">\n'.encode(),
           b"    </PDataArray>\n",
           f'    <PDataArray type="UInt8" Name="types" format="{fmt}">\n'.encode(),
           b"    </PDataArray>\n",
           b"   </PCells>\n"]
    for lv in range(levels):
        out.append(f'    <Piece Source="rank_0_grid_level_{lv}.vtu"/>\n'.encode())
    out.append(b" </PUnstructuredGrid>\n")
    out.append(b" </VTKFile>\n")
    return b"".join(out)


def parse_arrays(text: bytes) -> dict:
    """Name -> (type, components, raw numbers as a numpy array) of every DataArray of a .vtu."""
    import re
    s = text.decode()
    out = {}
    types = {"UInt16": np.uint16, "UInt8": np.uint8, "Float32": np.float32, "UInt64": np.uint64}
    for m in re.finditer(r'<DataArray([^>]*)>\n(.*?)\n?\s*</DataArray>', s, re.S):
        attrs = dict(re.findall(r'(\w+)="([^"]*)"', m.group(1)))
        name = attrs.get("Name", "Points")
        dt = types[attrs["type"]]
        body = m.group(2).strip()
        if attrs["format"] == "binary":
            raw = base64.b64decode(body)
            size = int.from_bytes(raw[:4], "little")
            arr = np.frombuffer(raw[4:4 + size], dtype=dt)
        else:
            arr = np.array(body.split(), dtype=np.float64 if dt == np.float32 else np.int64)
        out[name] = (attrs["type"], int(attrs.get("NumberOfComponents", 1)), arr)
    return out
