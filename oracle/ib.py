"""ORACLE — test infrastructure only.

Restatement of the immersed-boundary delta kernels and of the direct-forcing velocity
interpolation for the tests:
  * `delta_two`: the reference's four-point StencilDisTwo
    (lbm_project/immersed_boundary/immersed_boundary.cpp:365-384);
  * `delta_three`: the three-point kernel of Roma, Peskin and Berger (J. Comput. Phys. 153,
    1999), which the reference does not have;
  * `vertex_forces`: F = 2 (U_b - sum delta u) (immersed_boundary.cpp:183-184, :318-320) with
    the stencil placement of each width;
  * `spread`: node force += F delta area / (dt dx^(d-1)) over the same stencil
    (immersed_boundary.cpp:186-199, :322-339).
"""
from __future__ import annotations

import numpy as np


def delta_two(r):
    r = np.abs(np.asarray(r, dtype=np.float64))
    out = np.zeros_like(r)
    a = r < 1.0
    b = (r >= 1.0) & (r < 2.0)
    out[a] = 0.125 * (3.0 - 2.0 * r[a] + np.sqrt(1.0 + 4.0 * r[a] - 4.0 * r[a] ** 2))
    out[b] = 0.125 * (5.0 - 2.0 * r[b] - np.sqrt(-7.0 + 12.0 * r[b] - 4.0 * r[b] ** 2))
    return out


def delta_three(r):
    r = np.abs(np.asarray(r, dtype=np.float64))
    out = np.zeros_like(r)
    a = r <= 0.5
    b = (r > 0.5) & (r <= 1.5)
    out[a] = (1.0 + np.sqrt(1.0 - 3.0 * r[a] ** 2)) / 3.0
    out[b] = (5.0 - 3.0 * r[b] - np.sqrt(1.0 - 3.0 * (1.0 - r[b]) ** 2)) / 6.0
    return out


def stencil(x: float, width: int):
    """Node indices and weights along one axis for a point at x (grid units)."""
    if width == 4:
        idx = int(np.uint32(x + 1e-6))
        dis = x - float(np.uint32(x + 1e-6))
        nodes = np.arange(idx - 1, idx + 3)
        w = delta_two(np.array([dis - ix - 1 for ix in (-2, -1, 0, 1)]))
    else:
        j0 = int(np.floor(x + 0.5))
        nodes = np.arange(j0 - 1, j0 + 2)
        w = delta_three(x - nodes)
    return nodes, w


def vertex_forces(u_of, coords, vel, dx: float, width: int, dims: int = 2):
    """Vertex forces 2 (U_b - u(X)); u_of(ix, iy[, iz]) gives a node's velocity (level indices)."""
    out = np.zeros((len(coords), 3))
    for i, (c, ub) in enumerate(zip(coords, vel)):
        axes = [stencil(c[a] / dx, width) for a in range(dims)]
        acc = np.zeros(3)
        if dims == 2:
            for jy, wy in zip(*axes[1]):
                for jx, wx in zip(*axes[0]):
                    acc += u_of(jx, jy) * (wx * wy)
        else:
            for jz, wz in zip(*axes[2]):
                for jy, wy in zip(*axes[1]):
                    for jx, wx in zip(*axes[0]):
                        acc += u_of(jx, jy, jz) * (wx * wy * wz)
        out[i, :dims] = 2.0 * (np.asarray(ub[:dims]) - acc[:dims])
    return out


def spread(forces, coords, area, dx: float, dt: float, width: int, dims: int, add):
    """Share of every vertex force on its stencil nodes: add(node indices, share[3]) is called once
    per (vertex, stencil node), share = F * (delta * area / (dt dx^(d-1)))."""
    for c, force, a in zip(coords, forces, area):
        axes = [stencil(c[k] / dx, width) for k in range(dims)]
        scale = a / dt / dx if dims == 2 else a / dt / dx / dx
        force = np.asarray(force, dtype=np.float64)
        if dims == 2:
            for jy, wy in zip(*axes[1]):
                for jx, wx in zip(*axes[0]):
                    add((int(jx), int(jy)), force * (wx * wy * scale))
        else:
            for jz, wz in zip(*axes[2]):
                for jy, wy in zip(*axes[1]):
                    for jx, wx in zip(*axes[0]):
                        add((int(jx), int(jy), int(jz)), force * (wx * wy * wz * scale))
