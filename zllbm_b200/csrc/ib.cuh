// Immersed-boundary direct forcing on one level (FsiImmersedBoundary::CalculateBodyForce,
// lbm_project/immersed_boundary/immersed_boundary.cpp:35-364), split in three launches:
//   1. every node of every vertex stencil (each once, from a list built with the vertices) drops
//      its immersed-boundary force and records its velocity computed from the post-stream
//      populations with the remaining (constant) force (the reference does this on the first
//      touch of a node, :157-168);
//   2. every vertex interpolates the node velocities with the delta kernel and sets its force
//      F = 2 (U_b - u) (:183-184, :318-320);
//   3. every vertex spreads F delta area / (dt dx^(d-1)) into the node forces (:187-199, :322-339).
// The stencils of a vertex set are resolved once, when the vertices are set (ib_pairs_kernel):
// every (vertex, stencil node) pair gets its cell and FP64 delta weight, and every stencil node
// the list of its pairs in vertex order (a CSR built by a stable radix sort).  Launch 2 gives each
// vertex a warp that reads its pairs and sums with warp-shuffle reductions; launch 3 gives each
// stencil node a thread that sums the shares of its vertices in vertex order, so the spread needs
// no atomics and is deterministic.  Summation orders differ from the reference's (an unordered_map
// walk and a sequential stencil loop); sums agree to rounding.
//
// Stencils: width 4 is the reference's StencilDisTwo (immersed_boundary.cpp:365-384); width 3 is
// the three-point kernel of Roma, Peskin and Berger (J. Comput. Phys. 153, 1999), which the
// reference does not have.
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
    int width;            // stencil nodes per axis: 4 (reference) or 3 (Roma et al.)
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

// Three-point kernel (Roma, Peskin and Berger 1999): (1 + sqrt(1 - 3 r^2)) / 3 for |r| <= 1/2,
// (5 - 3 |r| - sqrt(1 - 3 (1 - |r|)^2)) / 6 for 1/2 <= |r| <= 3/2, zero beyond.
__device__ __forceinline__ double ib_delta_three(double dist) {
    const double a = fabs(dist);
    if (a <= 0.5) return (1. + sqrt(1. - 3. * a * a)) / 3.;
    if (a <= 1.5) {
        const double b = 1. - a;
        return (5. - 3. * a - sqrt(1. - 3. * b * b)) / 6.;
    }
    return 0.;
}

// Reference point of a vertex on axis a: the first stencil node `first` and the value whose
// distance to stencil node o is computed by ib_dist.  Width 4 keeps the reference's arithmetic
// (index (uint32)(r + 1e-6), distance |dis - ix - 1| with ix = o - 2); width 3 centres the stencil
// on the nearest node.
__device__ __forceinline__ void ib_reference(const IbVertices& v, const double* coord, int dims, long long* first,
                                             double* dis) {
    for (int a = 0; a < dims; ++a) {
        const double r = coord[a] / v.dx;
        if (v.width == 4) {
            const long long idx = (long long)(uint32_t)(r + 1e-6);
            first[a] = idx - 1;
            dis[a] = r - (double)(uint32_t)(r + 1e-6);
        } else {
            const long long j0 = (long long)floor(r + 0.5);
            first[a] = j0 - 1;
            dis[a] = r - (double)j0;
        }
    }
}

__device__ __forceinline__ double ib_weight(const IbVertices& v, double dis, int o) {
    if (v.width == 4) {
        const int ix = o - 2;
        return ib_delta_two(fabs(dis - ix - 1));
    }
    return ib_delta_three(dis - (double)(o - 1));
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

// Stencil node k of a vertex (k over width^dims nodes, x fastest): level indices and weight.
__device__ __forceinline__ double ib_stencil_node(const IbVertices& v, int dims, const long long* first,
                                                  const double* dis, int k, long long* nid) {
    const int w = v.width;
    const int o[3] = {k % w, (k / w) % w, k / (w * w)};
    double weight = 1.;
    for (int a = 0; a < 3; ++a) {
        if (a < dims) {
            nid[a] = first[a] + o[a];
            weight *= ib_weight(v, dis[a], o[a]);
        } else {
            nid[a] = 0;
        }
    }
    return weight;
}

// Every node a vertex stencil touches, once (the set is built when the vertices are set):
// launch 1 of the pass runs over this list rather than over (vertex, stencil node) pairs, which
// visit a node of the surface band once per vertex whose stencil holds it.
template <int D>
__global__ void ib_mark_kernel(LevelGeom geo, LevelMap m, IbVertices v, uint32_t* __restrict__ mark,
                               int* __restrict__ bad) {
    const int K = D == 3 ? v.width * v.width * v.width : v.width * v.width;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)v.n * K) return;
    const int i = (int)(t / K), k = (int)(t % K);
    long long first[3], nid[3];
    double dis[3];
    ib_reference(v, v.coord + i * 3, D, first, dis);
    ib_stencil_node(v, D, first, dis, k, nid);
    const long long cell = ib_cell(geo, m, nid, D);
    if (cell < 0) {
        atomicExch(bad, 1);
        return;
    }
    mark[cell] = 1u;
}

// A new vertex set (a body that moved): the nodes the previous set's stencils touched that the
// new set's stencils do not (all of them when mark is null) drop the force they last received.
// The reference resets only the nodes of the current stencils (immersed_boundary.cpp:157-167),
// which never differ from the previous ones because its shapes move no vertex.
static __global__ void ib_release_kernel(const int* __restrict__ nodes, int n_nodes,
                                         const uint32_t* __restrict__ mark, double* __restrict__ node_force) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_nodes) return;
    const long long cell = nodes[t];
    if (mark && mark[cell]) return;
    for (int a = 0; a < 3; ++a) node_force[cell * 3 + a] = 0.;
}

// Launch 1: the velocity of every stencil node (launch 3 then writes every stencil node's force),
// one array per component over the level's box cells (node_vel[a cells + cell]): a vertex's
// stencil rows are runs of consecutive cells, so the interpolation's loads of one component
// fall into few sectors.
template <class L, class S>
__global__ void ib_touch_kernel(const S* __restrict__ f, LevelGeom geo, StepParams p, int even_layout,
                                const int* __restrict__ nodes, int n_nodes, double* __restrict__ node_vel) {
    pdl_wait();
    pdl_trigger();
    using St = Storage<S>;
    using T = typename St::T;
    constexpr int Q = L::kQ, D = L::kDims;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_nodes) return;
    const long long cell = nodes[t];
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
    const long long cells = (long long)geo.a[0] * geo.a[1] * geo.a[2];
    for (int a = 0; a < 3; ++a) node_vel[a * cells + cell] = u[a];
}

// Every (vertex i, stencil node k) pair, k over width^D nodes x fastest: the node's cell, its
// index in the level's stencil-node list (the sort key of the CSR) and the delta weight, formed as
// ib_stencil_node forms it (the 1-D weights multiplied in axis order).  Runs when the vertices are set.
template <int D>
__global__ void ib_pairs_kernel(LevelGeom geo, LevelMap m, IbVertices v, const int* __restrict__ node_of_cell,
                                int* __restrict__ pair_cell, double* __restrict__ pair_w, int* __restrict__ pair_node,
                                int* __restrict__ pair_id) {
    const int K = D == 3 ? v.width * v.width * v.width : v.width * v.width;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)v.n * K) return;
    const int i = (int)(t / K), k = (int)(t % K);
    long long first[3], nid[3];
    double dis[3];
    ib_reference(v, v.coord + i * 3, D, first, dis);
    const double w = ib_stencil_node(v, D, first, dis, k, nid);
    const long long cell = ib_cell(geo, m, nid, D);  // present: checked by ib_mark_kernel
    pair_cell[t] = (int)cell;
    pair_w[t] = w;
    pair_node[t] = node_of_cell[cell];
    pair_id[t] = (int)t;
}

// Launch 2: kIbForceLanes lanes per vertex interpolate the node velocities through its pairs (a
// vertex has 64 pairs in 3D, 16 in 2D with the four-point kernel): lane k takes pairs k,
// k + kIbForceLanes, ..., four at a time with their loads issued first (one round of two dependent
// loads for the 3D kernel) and summed two by two, and the lanes' sums are combined by a fixed
// butterfly of shuffles.  The first lane writes F = 2 (U_b - sum delta u).
constexpr int kIbForceLanes = 16;
constexpr int kIbForceThreads = 128;

template <int D>
__global__ void __launch_bounds__(kIbForceThreads) ib_force_kernel(IbVertices v, const int* __restrict__ pair_cell,
                                                                   const double* __restrict__ pair_w,
                                                                   const double* __restrict__ node_vel,
                                                                   long long cells) {
    pdl_wait();
    pdl_trigger();
    constexpr int G = kIbForceLanes;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int i = (int)(t / G), lane = (int)(t % G);
    const bool live = i < v.n;  // every lane of the warp takes part in the shuffles
    double u[3] = {0., 0., 0.};
    if (live) {
        const int K = D == 3 ? v.width * v.width * v.width : v.width * v.width;
        const long long base = (long long)i * K;
        int k = lane;
        for (; k + 3 * G < K; k += 4 * G) {
            long long c[4];
            double d[4], a[4][3];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                c[e] = __ldg(pair_cell + base + k + e * G);
                d[e] = __ldg(pair_w + base + k + e * G);
            }
#pragma unroll
            for (int e = 0; e < 4; ++e)
#pragma unroll
                for (int b = 0; b < D; ++b) a[e][b] = node_vel[b * cells + c[e]];
#pragma unroll
            for (int b = 0; b < D; ++b) u[b] = u[b] + a[0][b] * d[0] + a[1][b] * d[1];
#pragma unroll
            for (int b = 0; b < D; ++b) u[b] = u[b] + a[2][b] * d[2] + a[3][b] * d[3];
        }
        for (; k + G < K; k += 2 * G) {
            const long long c0 = __ldg(pair_cell + base + k), c1 = __ldg(pair_cell + base + k + G);
            const double d0 = __ldg(pair_w + base + k), d1 = __ldg(pair_w + base + k + G);
            double a0[3], a1[3];
#pragma unroll
            for (int a = 0; a < D; ++a) {
                a0[a] = node_vel[a * cells + c0];
                a1[a] = node_vel[a * cells + c1];
            }
#pragma unroll
            for (int a = 0; a < D; ++a) u[a] = u[a] + a0[a] * d0 + a1[a] * d1;
        }
        if (k < K) {
            const long long c = __ldg(pair_cell + base + k);
            const double d = __ldg(pair_w + base + k);
#pragma unroll
            for (int a = 0; a < D; ++a) u[a] += node_vel[a * cells + c] * d;
        }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1)
#pragma unroll
        for (int a = 0; a < D; ++a) u[a] += __shfl_xor_sync(0xffffffffu, u[a], o);
    if (!live || lane) return;
    v.force[i * 3] = 2. * (v.vel[i * 3] - u[0]);
    v.force[i * 3 + 1] = 2. * (v.vel[i * 3 + 1] - u[1]);
    v.force[i * 3 + 2] = D == 3 ? 2. * (v.vel[i * 3 + 2] - u[2]) : 0.;
}

// Launch 3: kIbSpreadLanes lanes per stencil node sum F_i s_p over the node's pairs p (vertex i):
// lane k takes pairs k, k + kIbSpreadLanes, ... of the node's CSR row, two at a time with their
// loads issued first, and the lanes' sums are combined by a fixed butterfly of shuffles
// (deterministic).  The first lane writes the node force (every stencil node owns at least one
// pair, so every node of the list is written; no other pass adds to it).  s_p = delta_p area_i / (dt dx^(d-1)) and the vertex index come from the CSR arrays,
// laid out in node order.  A node has about 16 (3D) pairs: the lanes cut the chain of dependent
// loads per thread eightfold and give the launch eight times the threads.
constexpr int kIbSpreadLanes = 8;

template <int D>
__global__ void ib_spread_kernel(IbVertices v, const int* __restrict__ nodes, int n_nodes,
                                 const int* __restrict__ csr_start, const int* __restrict__ csr_vertex,
                                 const double* __restrict__ csr_share, double* __restrict__ node_force) {
    pdl_wait();
    pdl_trigger();
    constexpr int G = kIbSpreadLanes;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int j = (int)(t / G), k = (int)(t % G);
    const bool live = j < n_nodes;  // every lane of the warp takes part in the shuffles
    double F[3] = {0., 0., 0.};
    if (live) {
        const int s1 = csr_start[j + 1];
        int s = csr_start[j] + k;
        for (; s + G < s1; s += 2 * G) {
            const int i0 = __ldg(csr_vertex + s), i1 = __ldg(csr_vertex + s + G);
            const double h0 = __ldg(csr_share + s), h1 = __ldg(csr_share + s + G);
            double f0[3], f1[3];
#pragma unroll
            for (int a = 0; a < D; ++a) {
                f0[a] = v.force[i0 * 3 + a];
                f1[a] = v.force[i1 * 3 + a];
            }
#pragma unroll
            for (int a = 0; a < D; ++a) F[a] = F[a] + f0[a] * h0 + f1[a] * h1;
        }
        if (s < s1) {
            const int i = __ldg(csr_vertex + s);
            const double h = __ldg(csr_share + s);
#pragma unroll
            for (int a = 0; a < D; ++a) F[a] += v.force[i * 3 + a] * h;
        }
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1)
#pragma unroll
        for (int a = 0; a < D; ++a) F[a] += __shfl_xor_sync(0xffffffffu, F[a], off);
    if (!live || k) return;
    const long long cell = nodes[j];
    for (int a = 0; a < D; ++a) node_force[cell * 3 + a] = F[a];
}

// The spread CSR in node order: for sorted position t the vertex of pair csr_pair[t] and its share
// delta area / (dt dx^(d-1)), with the division order of the direct formula.  Runs with the vertices.
template <int D>
__global__ void ib_csr_fill_kernel(IbVertices v, double dt, const int* __restrict__ csr_pair,
                                   const double* __restrict__ pair_w, long long pairs, int* __restrict__ csr_vertex,
                                   double* __restrict__ csr_share) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= pairs) return;
    const int K = D == 3 ? v.width * v.width * v.width : v.width * v.width;
    const int pr = csr_pair[t];
    const int i = pr / K;
    const double area = D == 3 ? v.area[i] / dt / v.dx / v.dx : v.area[i] / dt / v.dx;
    csr_vertex[t] = i;
    csr_share[t] = pair_w[pr] * area;
}

// CSR row starts of the sorted pair keys (every stencil node owns at least one pair).
static __global__ void ib_csr_start_kernel(const int* __restrict__ sorted_node, long long pairs,
                                           int* __restrict__ start, int n_nodes) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t > pairs) return;
    if (t == pairs) {
        start[n_nodes] = (int)pairs;
        return;
    }
    if (t == 0 || sorted_node[t] != sorted_node[t - 1]) start[sorted_node[t]] = (int)t;
}

// node_of_cell[nodes[j]] = j over the level's stencil-node list.
static __global__ void ib_index_nodes_kernel(const int* __restrict__ nodes, int n_nodes, int* __restrict__ node_of_cell) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n_nodes) node_of_cell[nodes[j]] = j;
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
