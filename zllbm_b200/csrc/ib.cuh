// Immersed-boundary direct forcing on one level (FsiImmersedBoundary::CalculateBodyForce,
// lbm_project/immersed_boundary/immersed_boundary.cpp:35-364), split in three launches:
//   1. every node of every vertex stencil drops its immersed-boundary force and records its
//      velocity computed from the post-stream populations with the remaining (constant) force
//      (the reference does this on the first touch of a node, :157-168);
//   2. every vertex interpolates the node velocities with the delta kernel and sets its force
//      F = 2 (U_b - u) (:183-184, :318-320);
//   3. every vertex spreads F delta area / (dt dx^(d-1)) into the node forces (:187-199, :322-339).
// Launch 3 accumulates with FP64 atomics, so the order in which vertices add into a node is not
// fixed; the reference's order is that of an unordered_map.  Sums agree to rounding.
#pragma once
#include "level_ops.cuh"

namespace zl {

struct IbVertices {
    const double* coord;  // n * 3, the reference's vertex coordinate_ (domain offset included)
    const double* vel;    // n * 3, vertex velocity_
    const double* area;   // n, vertex area_ (arc length in 2D)
    double* force;        // n * 3, vertex force_ (written by launch 2)
    int n;
    double dx;            // grid spacing of the level
};

// Stencil of the delta kernel (StencilDisOne / StencilDisTwo, immersed_boundary.cpp:365-384)
__device__ __forceinline__ double ib_delta_two(double dist) {
    if (dist < 2.) {
        const double a = fabs(dist);
        const double sq = dist * dist;
        if (a < 1.) return 0.125 * (3. - 2. * a + sqrt(1. + 4. * a - 4. * sq));
        return 0.125 * (5. - 2. * a - sqrt(-7. + 12. * a - 4. * sq));
    }
    return 0.;
}

// Reference point of a vertex: level indices and the fractional distances.
__device__ __forceinline__ void ib_reference(const IbVertices& v, int i, int dims, long long* idx, double* dis) {
    for (int a = 0; a < dims; ++a) {
        const double r = v.coord[i * 3 + a] / v.dx;
        idx[a] = (long long)(uint32_t)(r + 1e-6);
        dis[a] = r - (double)(uint32_t)(r + 1e-6);
    }
}

// Node cell of level indices, -1 when the node is not on the level.
__device__ __forceinline__ long long ib_cell(const LevelGeom& geo, const LevelMap& m, const long long* idx, int dims) {
    long long b[3] = {0, 0, 0};
    for (int a = 0; a < dims; ++a) {
        long long x = idx[a] - m.lo[a];
        if (m.periodic[a]) x = ((x % m.n[a]) + m.n[a]) % m.n[a];
        if (x < 0 || x >= m.n[a]) return -1;
        b[a] = x + geo.g[a];
    }
    const long long cell = b[0] + (long long)geo.a[0] * (b[1] + (long long)geo.a[1] * b[2]);
    if (geo.info && !(__ldg(geo.info + cell) & kInfoPresent)) return -1;
    return cell;
}

template <class L, class S>
__global__ void ib_touch_kernel(const S* __restrict__ f, LevelGeom geo, LevelMap m, StepParams p, int even_layout,
                                IbVertices v, double* __restrict__ node_force, double* __restrict__ node_vel,
                                int* __restrict__ bad) {
    using St = Storage<S>;
    using T = typename St::T;
    constexpr int Q = L::kQ, D = L::kDims;
    constexpr int K = D == 3 ? 64 : 16;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= v.n * K) return;
    const int i = t / K, k = t % K;
    long long idx[3], nid[3];
    double dis[3];
    ib_reference(v, i, D, idx, dis);
    nid[0] = idx[0] + (k & 3) - 1;
    nid[1] = idx[1] + ((k >> 2) & 3) - 1;
    nid[2] = D == 3 ? idx[2] + ((k >> 4) & 3) - 1 : 0;
    const long long cell = ib_cell(geo, m, nid, D);
    if (cell < 0) {
        atomicExch(bad, 1);
        return;
    }
    Coord c = cell_coord(geo, (int)cell);
    T fv[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) fv[q] = St::load(f + post_stream_slot<L>(geo, c, q, even_layout), p);
    // func_macro_with_force_ with the node's immersed-boundary force set to zero
    double u[3];
    if constexpr (St::kDeviation) {
        float rho, ux, uy, uz;
        macro_dev<L>(fv, rho, ux, uy, uz);
        const double h = 0.5 * p.dt / rho;
        u[0] = ux + h * p.const_force[0];
        u[1] = uy + h * p.const_force[1];
        u[2] = uz + h * p.const_force[2];
    } else {
        using Tb = Tables<L>;
        double rho = fv[0], ux = 0., uy = 0., uz = 0.;
#pragma unroll
        for (int q = 1; q < Q; ++q) {
            rho = rho + fv[q];
            if (Tb::cx(q) == 1) ux = ux + fv[q];
            if (Tb::cx(q) == -1) ux = ux - fv[q];
            if (Tb::cy(q) == 1) uy = uy + fv[q];
            if (Tb::cy(q) == -1) uy = uy - fv[q];
            if (D == 3) {
                if (Tb::cz(q) == 1) uz = uz + fv[q];
                if (Tb::cz(q) == -1) uz = uz - fv[q];
            }
        }
        ux = ux + 0.5 * p.const_force[0] * p.dt;
        uy = uy + 0.5 * p.const_force[1] * p.dt;
        if (D == 3) uz = uz + 0.5 * p.const_force[2] * p.dt;
        u[0] = ux / rho;
        u[1] = uy / rho;
        u[2] = D == 3 ? uz / rho : 0.;
    }
    for (int a = 0; a < 3; ++a) {
        node_force[cell * 3 + a] = 0.;
        node_vel[cell * 3 + a] = u[a];
    }
}

template <int D>
__global__ void ib_force_kernel(LevelGeom geo, LevelMap m, IbVertices v, const double* __restrict__ node_vel) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= v.n) return;
    long long idx[3];
    double dis[3];
    ib_reference(v, i, D, idx, dis);
    double ur = 0., vr = 0., wr = 0.;
    const int nz = D == 3 ? 4 : 1;
    for (int iz = -2; iz < -2 + nz; ++iz) {
        const double dz = D == 3 ? ib_delta_two(fabs(dis[2] - iz - 1)) : 1.;
        for (int iy = -2; iy < 2; ++iy) {
            const double dy = ib_delta_two(fabs(dis[1] - iy - 1));
            for (int ix = -2; ix < 2; ++ix) {
                const double dx = ib_delta_two(fabs(dis[0] - ix - 1));
                const long long nid[3] = {idx[0] + ix + 1, idx[1] + iy + 1, D == 3 ? idx[2] + iz + 1 : 0};
                const long long cell = ib_cell(geo, m, nid, D);
                const double delta = D == 3 ? dx * dy * dz : dx * dy;
                ur += node_vel[cell * 3] * delta;
                vr += node_vel[cell * 3 + 1] * delta;
                if (D == 3) wr += node_vel[cell * 3 + 2] * delta;
            }
        }
    }
    v.force[i * 3] = 2. * (v.vel[i * 3] - ur);
    v.force[i * 3 + 1] = 2. * (v.vel[i * 3 + 1] - vr);
    v.force[i * 3 + 2] = D == 3 ? 2. * (v.vel[i * 3 + 2] - wr) : 0.;
}

template <int D>
__global__ void ib_spread_kernel(LevelGeom geo, LevelMap m, StepParams p, IbVertices v,
                                 double* __restrict__ node_force) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= v.n) return;
    long long idx[3];
    double dis[3];
    ib_reference(v, i, D, idx, dis);
    const double area = D == 3 ? v.area[i] / p.dt / v.dx / v.dx : v.area[i] / p.dt / v.dx;
    const int nz = D == 3 ? 4 : 1;
    for (int iz = -2; iz < -2 + nz; ++iz) {
        const double dz = D == 3 ? ib_delta_two(fabs(dis[2] - iz - 1)) : 1.;
        for (int iy = -2; iy < 2; ++iy) {
            const double dy = ib_delta_two(fabs(dis[1] - iy - 1));
            for (int ix = -2; ix < 2; ++ix) {
                const double dx = ib_delta_two(fabs(dis[0] - ix - 1));
                const long long nid[3] = {idx[0] + ix + 1, idx[1] + iy + 1, D == 3 ? idx[2] + iz + 1 : 0};
                const long long cell = ib_cell(geo, m, nid, D);
                const double dt = (D == 3 ? dx * dy * dz : dx * dy) * area;
                for (int a = 0; a < D; ++a) atomicAdd(node_force + cell * 3 + a, v.force[i * 3 + a] * dt);
            }
        }
    }
}

// Sum over vertices of F area / dx_background^(d-1) in vertex order (WriteTimeHisLagrangianForce,
// immersed_boundary.cpp:596-642), FP64, one thread.
static __global__ void ib_total_kernel(IbVertices v, double scale, double* __restrict__ out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double fx = 0., fy = 0., fz = 0.;
    for (int i = 0; i < v.n; ++i) {
        fx += v.force[i * 3] * v.area[i] * scale;
        fy += v.force[i * 3 + 1] * v.area[i] * scale;
        fz += v.force[i * 3 + 2] * v.area[i] * scale;
    }
    out[0] = fx;
    out[1] = fy;
    out[2] = fz;
}

}  // namespace zl
