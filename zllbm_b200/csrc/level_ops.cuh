// Per-level kernels other than the fused step: non-equilibrium extrapolation
// faces, host <-> device population exchange in the reference's node order,
// macroscopic fields and FP64 conservation sums.
#pragma once
#include "aa_kernel.cuh"

namespace zl {

// Mapping from a reference Morton code to this level's node coordinates.
struct LevelMap {
    int dims;
    int lo[3];        // reference index of node coordinate 0 (at this level)
    int n[3];
    int periodic[3];  // a periodic axis stores the max plane folded onto coordinate 0
};

// Bit-exact restatement of SFBitsetComputeIndices (amr_project/grid/morton_aux.cpp:107-119, :336-351).
ZL_HD void morton_decode(uint64_t code, int dims, uint32_t* idx) {
    idx[0] = idx[1] = idx[2] = 0;
    const int nbits = 64 / dims;
    for (int i = 0; i < nbits; ++i)
        for (int a = 0; a < dims; ++a) idx[a] |= (uint32_t)((code >> (dims * i + a)) & 1ull) << i;
}

ZL_HD uint64_t morton_encode(const uint32_t* idx, int dims) {
    uint64_t code = 0;
    const int nbits = 64 / dims;
    for (int i = 0; i < nbits; ++i)
        for (int a = 0; a < dims; ++a) code |= (uint64_t)((idx[a] >> i) & 1u) << (dims * i + a);
    return code;
}

// `folded` (optional) is set when the code lies on the duplicated maximum plane of a periodic
// axis and was folded onto coordinate 0.
__device__ __forceinline__ bool code_to_node(uint64_t code, const LevelMap& m, Coord& c, bool* folded = nullptr) {
    uint32_t idx[3];
    morton_decode(code, m.dims, idx);
    c.x[2] = 0;
    bool fold = false;
    for (int a = 0; a < m.dims; ++a) {
        int v = (int)idx[a] - m.lo[a];
        if (m.periodic[a] && v == m.n[a]) {
            v = 0;
            fold = true;
        }
        if (v < 0 || v >= m.n[a]) return false;
        c.x[a] = v;
    }
    if (folded) *folded = fold;
    return true;
}

// Node coordinates of a box cell index (inverse of the box indexing, ghost frame removed).
__device__ __forceinline__ Coord cell_coord(const LevelGeom& geo, int cell) {
    Coord c;
    const uint32_t u = (uint32_t)cell, rest = geo.fa0.div(u), bz = geo.fa1.div(rest);
    const int bx = (int)(u - rest * (uint32_t)geo.a[0]);
    const int by = (int)(rest - bz * (uint32_t)geo.a[1]);
    c.x[0] = bx - geo.g[0];
    c.x[1] = by - geo.g[1];
    c.x[2] = bz - geo.g[2];
    return c;
}

// ---------------------------------------------------------------- deviation-form helpers
template <class L>
__device__ __forceinline__ void macro_dev(const float* d, float& rho, float& ux, float& uy, float& uz) {
    using Tb = Tables<L>;
    float drho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int q = 0; q < L::kQ; ++q) {
        drho += d[q];
        if (Tb::cx(q)) jx += Tb::cx(q) == 1 ? d[q] : -d[q];
        if (Tb::cy(q)) jy += Tb::cy(q) == 1 ? d[q] : -d[q];
        if (L::kDims == 3 && Tb::cz(q)) jz += Tb::cz(q) == 1 ? d[q] : -d[q];
    }
    rho = 1.f + drho;
    ux = jx / rho;
    uy = jy / rho;
    uz = jz / rho;
}

template <class L>
__device__ __forceinline__ void feq_dev(float rho, float ux, float uy, float uz, float* deq) {
    using Tb = Tables<L>;
    const float usq15 = 1.5f * (ux * ux + uy * uy + uz * uz);
#pragma unroll
    for (int q = 0; q < L::kQ; ++q) {
        const float cu = signed_dot<L>(q, ux, uy, uz);
        deq[q] = (float)Tb::w(q) * ((rho - 1.f) + rho * (3.f * cu + 4.5f * cu * cu - usq15));
    }
}

// ---------------------------------------------------------------- NEQ extrapolation
// lbm_project/boundary_conditions/lbm_noneq_extrapolation.cpp:89-144: every population of a
// face node becomes feq(rho0, U_face) + f(inner) - feq(rho(inner), u(inner)), using the inner
// node's post-stream populations.  One launch per face, in the reference's face order.
template <class L, class S>
__global__ void neq_face_kernel(S* __restrict__ f, LevelGeom geo, StepParams p, int face, int even_layout,
                                const double* __restrict__ feq_b) {
    pdl_wait();
    pdl_trigger();
    using St = Storage<S>;
    using T = typename St::T;
    constexpr int Q = L::kQ;
    const int axis = face >> 1;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;  // coordinate along first other axis
    const int t1 = blockIdx.y;                             // along second other axis (3D)
    const int o0 = axis == 0 ? 1 : 0;
    const int o1 = axis == 2 ? 1 : 2;
    if (t0 >= geo.n[o0]) return;
    if (L::kDims == 3 && t1 >= geo.n[o1]) return;
    Coord c;
    c.x[2] = 0;
    c.x[axis] = (face & 1) ? geo.n[axis] - 1 : 0;
    c.x[o0] = t0;
    if (L::kDims == 3) c.x[o1] = t1;
    const long long self = (long long)(c.x[0] + geo.g[0]) +
                           (long long)geo.a[0] * ((c.x[1] + geo.g[1]) + (long long)geo.a[1] * (c.x[2] + geo.g[2]));
    if (geo.info && !(__ldg(geo.info + self) & kInfoPresent)) return;
    Coord ci = c;
    ci.x[axis] += (face & 1) ? -1 : 1;
    if (geo.info) {
        const long long inner = (long long)(ci.x[0] + geo.g[0]) +
                                (long long)geo.a[0] * ((ci.x[1] + geo.g[1]) + (long long)geo.a[1] * (ci.x[2] + geo.g[2]));
        if (!(__ldg(geo.info + inner) & kInfoPresent)) return;
    }
    T fi[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) fi[q] = St::load(f + post_stream_slot<L>(geo, ci, q, even_layout), p);
    // inner node macros through func_macro_ (with the node's forces when the solver has forces)
    double F[3] = {0., 0., 0.};
    if (p.forced) {
        const long long inner = (long long)(ci.x[0] + geo.g[0]) +
                                (long long)geo.a[0] * ((ci.x[1] + geo.g[1]) + (long long)geo.a[1] * (ci.x[2] + geo.g[2]));
        for (int a = 0; a < 3; ++a) F[a] = p.const_force[a] + (p.force ? p.force[inner * 3 + a] : 0.);
    }
    if constexpr (St::kDeviation) {
        float rho, ux, uy, uz, deq[Q];
        macro_dev<L>(fi, rho, ux, uy, uz);
        if (p.forced) {
            const float h = 0.5f * (float)p.dt / rho;
            ux += h * (float)F[0];
            uy += h * (float)F[1];
            uz += h * (float)F[2];
        }
        feq_dev<L>(rho, ux, uy, uz, deq);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float db = (float)(feq_b[q] - Tables<L>::w(q));
            St::store(f + post_stream_slot<L>(geo, c, q, even_layout), db + fi[q] - deq[q], p);
        }
    } else {
        double rho, ux, uy, uz, feq[Q];
        macro_exact<L>(fi, rho, ux, uy, uz, p.forced ? F : nullptr, p.dt);
        feq_exact<L>(rho, ux, uy, uz, feq);
#pragma unroll
        for (int q = 0; q < Q; ++q)
            St::store(f + post_stream_slot<L>(geo, c, q, even_layout), (feq_b[q] + fi[q]) - feq[q], p);
    }
}

// ---------------------------------------------------------------- ordered face passes
// Face nodes of `face` (the box edge lying on that domain face), one thread each.
struct FaceNode {
    Coord c;
    long long self;
    bool ok;
};

template <class L>
__device__ __forceinline__ FaceNode face_node(const LevelGeom& geo, int face) {
    FaceNode r;
    const int axis = face >> 1;
    const int o0 = axis == 0 ? 1 : 0;
    const int o1 = axis == 2 ? 1 : 2;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int t1 = blockIdx.y;
    r.ok = t0 < geo.n[o0] && (L::kDims == 2 || t1 < geo.n[o1]);
    r.c.x[2] = 0;
    r.c.x[axis] = (face & 1) ? geo.n[axis] - 1 : 0;
    r.c.x[o0] = t0;
    if (L::kDims == 3) r.c.x[o1] = t1;
    r.self = (long long)(r.c.x[0] + geo.g[0]) +
             (long long)geo.a[0] * ((r.c.x[1] + geo.g[1]) + (long long)geo.a[1] * (r.c.x[2] + geo.g[2]));
    if (r.ok && geo.info && !(__ldg(geo.info + r.self) & kInfoPresent)) r.ok = false;
    return r;
}

// Convective outflow (no counterpart in the reference, which only has bounce back, periodic and
// non-equilibrium extrapolation faces): every population entering the domain across the face is
// advected out of the inner node with speed U (a first-order upwind step of df/dt + U df/dn = 0),
//     f(x_b, q) = (f_old(x_b, q) + U f(x_b - n, q)) / (1 + U),
// where f_old is the stale value the stream left at x_b and f(x_b - n, q) the inner node's new
// post-stream value.  The formula is linear, so deviation and scaled storage use it unchanged.
template <class L, class S>
__global__ void conv_face_kernel(S* __restrict__ f, LevelGeom geo, StepParams p, int face, int even_layout) {
    pdl_wait();
    pdl_trigger();
    using St = Storage<S>;
    using Tb = Tables<L>;
    using T = typename St::T;
    const FaceNode r = face_node<L>(geo, face);
    if (!r.ok) return;
    const int axis = face >> 1;
    const int out = (face & 1) ? 1 : -1;  // outward normal along the axis
    Coord ci = r.c;
    ci.x[axis] -= out;
    if (geo.info) {
        const long long inner = (long long)(ci.x[0] + geo.g[0]) +
                                (long long)geo.a[0] * ((ci.x[1] + geo.g[1]) + (long long)geo.a[1] * (ci.x[2] + geo.g[2]));
        if (!(__ldg(geo.info + inner) & kInfoPresent)) return;
    }
    const T u = (T)p.conv_u[face];
    const T one = (T)1;
#pragma unroll
    for (int q = 1; q < L::kQ; ++q) {
        const int ca = axis == 0 ? Tb::cx(q) : (axis == 1 ? Tb::cy(q) : Tb::cz(q));
        if (ca * out >= 0) continue;  // enters across this face iff c . n_out < 0
        const long long sb = post_stream_slot<L>(geo, r.c, q, even_layout);
        const T fb = St::load_raw(f + sb);
        const T fi = St::load_raw(f + post_stream_slot<L>(geo, ci, q, even_layout));
        St::store_raw(f + sb, (fb + u * fi) / (one + u));
    }
}

// Bounce back as its own pass (lbm_bounce_back.cpp:28-91): f(x, q_in) = f*(x, o) - 6 rho0 w_o (c_o.U),
// o = bb_source(q_in, face).
// Used when the level's faces must be applied one after another in the reference's order.
template <class L, class S>
__global__ void bb_face_kernel(S* __restrict__ f, LevelGeom geo, StepParams p, int face, int even_layout) {
    pdl_wait();
    pdl_trigger();
    using St = Storage<S>;
    const FaceNode fn = face_node<L>(geo, face);
    if (!fn.ok) return;
#pragma unroll
    for (int q = 1; q < L::kQ; ++q) {
        if (!enters_through<L>(q, face)) continue;
        const int o = bb_source<L>(q, face);
        const auto v = St::load(f + post_collision_slot<L>(geo, fn.c, o, even_layout), p);
        St::store(f + post_stream_slot<L>(geo, fn.c, q, even_layout), v - (decltype(v))p.bb_term[face][o], p);
    }
}

// Periodic face on a level that keeps the reference's duplicated maximum plane
// (lbm_periodic.cpp:77-133): the populations entering through the face are copied from the
// node with the same other coordinates on the opposite face.
template <class L, class S>
__global__ void periodic_face_kernel(S* __restrict__ f, LevelGeom geo, StepParams p, int face, int even_layout) {
    pdl_wait();
    pdl_trigger();
    using St = Storage<S>;
    const FaceNode fn = face_node<L>(geo, face);
    if (!fn.ok) return;
    const int axis = face >> 1;
    Coord other = fn.c;
    other.x[axis] = (face & 1) ? 0 : geo.n[axis] - 1;
    if (geo.info) {
        const long long oc = (long long)(other.x[0] + geo.g[0]) +
                             (long long)geo.a[0] * ((other.x[1] + geo.g[1]) + (long long)geo.a[1] * (other.x[2] + geo.g[2]));
        if (!(__ldg(geo.info + oc) & kInfoPresent)) return;
    }
#pragma unroll
    for (int q = 1; q < L::kQ; ++q) {
        if (!enters_through<L>(q, face)) continue;
        St::store(f + post_stream_slot<L>(geo, fn.c, q, even_layout),
                  St::load(f + post_stream_slot<L>(geo, other, q, even_layout), p), p);
    }
}

// ---------------------------------------------------------------- coarse <-> fine transfer
// Interpolation stencil of one fine ghost node: entries [offset[t], offset[t+1]) of the source
// arrays, in the reference's loop order (z outer, x inner, grid/grid_interpolation.cpp:485-517).
// Every distinct source node is evaluated once per transfer (c2f_sources_kernel) into the
// table g; the targets then form their weighted sums from the table.
constexpr int kC2fThreads = 128;  // explosion kernel block

struct C2FStencil {
    const int* target;        // fine cell of every target node
    const int* offset;        // n_targets + 1
    const int* src;           // entry -> row of the source table
    const double* weight;
    const int2* src_w32;      // (src, FP32 bits of the weight) per entry (FP32 / FP16 / BF16 storage)
    int n_targets;
    const int* src_cell;      // per source: coarse cell (src_fine == 0) or fine cell (src_fine == 1)
    const uint8_t* src_fine;
    int n_sources;
    void* g;                  // n_sources rows of c2f_row values (the storage's arithmetic type)
};

// The source table's rows: Q values in FP64; in FP32, Q values and zeros up to a whole number of
// float4 groups, so that a lane reads four populations of a source in one 16-byte load.
template <class L, class T>
ZL_HD constexpr int c2f_row() {
    return sizeof(T) == 8 ? L::kQ : 4 * ((L::kQ + 3) / 4);
}
// Threads per explosion target: one per population in FP64, one per float4 group in FP32.
template <class L, class T>
ZL_HD constexpr int c2f_lanes() {
    return sizeof(T) == 8 ? L::kQ : (L::kQ + 3) / 4;
}

// Explosion (TransferInfoFromCoarseGrid, lbm_grid_interface.cpp:408-515): every fine ghost node
// becomes sum_k w_k g_k with g_k = feq(rho_c, u_c) + tau_c2f (f_c - feq) for a coarse source
// (NodeInfoCoarse2fine + PostStreamCoarse2Fine, lbm_grid_interface.cpp:570-588,
// collision_model/lbm_collision_models.cpp:244-251) or the post-stream populations of the
// coincident fine node when the coarse node is absent or flagged.
// One thread per distinct source: g = feq(rho_c, u_c) + tau_c2f (f_c - feq) for a coarse source,
// the post-stream populations for a fine one.
template <class L, class S>
__global__ void c2f_sources_kernel(const S* __restrict__ ff, LevelGeom fgeo, int f_even, const S* __restrict__ fc,
                                   LevelGeom cgeo, int c_even, StepParams fp, StepParams cp, C2FStencil st,
                                   double tau_ratio) {
    pdl_wait();
    pdl_trigger();
    using St = Storage<S>;
    using T = typename St::T;
    constexpr int Q = L::kQ;
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= st.n_sources) return;
    T g[Q];
    if (st.src_fine[u]) {
        const Coord c = cell_coord(fgeo, st.src_cell[u]);
#pragma unroll
        for (int q = 0; q < Q; ++q) g[q] = St::load(ff + post_stream_slot<L>(fgeo, c, q, f_even), fp);
    } else {
        const Coord c = cell_coord(cgeo, st.src_cell[u]);
        T fcq[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) fcq[q] = St::load(fc + post_stream_slot<L>(cgeo, c, q, c_even), cp);
        if constexpr (St::kDeviation) {
            float rho, ux, uy, uz, deq[Q];
            macro_dev<L>(fcq, rho, ux, uy, uz);
            feq_dev<L>(rho, ux, uy, uz, deq);
#pragma unroll
            for (int q = 0; q < Q; ++q) g[q] = deq[q] + (float)tau_ratio * (fcq[q] - deq[q]);
        } else {
            double rho, ux, uy, uz, feq[Q];
            macro_exact<L>(fcq, rho, ux, uy, uz);
            feq_exact<L>(rho, ux, uy, uz, feq);
#pragma unroll
            for (int q = 0; q < Q; ++q) g[q] = feq[q] + tau_ratio * (fcq[q] - feq[q]);
        }
    }
    constexpr int R = c2f_row<L, T>();
    T* out = static_cast<T*>(st.g) + (long long)u * R;
    if constexpr (sizeof(T) == 4) {
        // the FP32 row as float4 stores (a quarter of the store requests; the kernel is bound by
        // its stores, one row per thread)
        float v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = q < Q ? g[q] : 0.f;
        float4* o4 = reinterpret_cast<float4*>(out);
#pragma unroll
        for (int j = 0; j < R / 4; ++j) o4[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) out[q] = g[q];
    }
}

// Explosion (TransferInfoFromCoarseGrid, lbm_grid_interface.cpp:408-515): every fine ghost node
// becomes sum_k w_k g_k over its sources in the reference's order, g_k from the source table
// (NodeInfoCoarse2fine + PostStreamCoarse2Fine, lbm_grid_interface.cpp:570-588,
// collision_model/lbm_collision_models.cpp:244-251, or the post-stream populations of the
// coincident fine node when the coarse node is absent or flagged).
// save (optional) receives the targets' values (n_targets x Q, in the storage's arithmetic type:
// FP64 for FP64 storage, FP32 otherwise); with prev (optional) the targets get 0.5 (prev + value)
// instead, the time interpolation between the last transfer and the coarse level's current state
// (no counterpart in the reference, whose explosion is spatial only); store = 0 only saves.
// FP64: one thread per (target, population q), consecutive threads taking consecutive q of a
// target: every lane of a warp works (Q = 19 or 9 does not divide a warp), the target's source
// indices and weights are loads the target's lanes share, and the source rows are read coalesced.
// FP32: one thread per (target, group of four populations), each source row read as one float4
// per thread (a quarter of the load requests: the kernel is bound by the L1 requests of its
// gathers).  Each thread sums over the target's sources in table order, every population in the
// same order as the one-population form (FP64 keeps its summation order), four sources' loads in
// flight at a time.
template <class L, class S>
__device__ __forceinline__ void c2f_thread(long long i, S* __restrict__ ff, const LevelGeom& fgeo, int f_even,
                                           const StepParams& fp, const C2FStencil& st,
                                           typename Storage<S>::T* __restrict__ save,
                                           const typename Storage<S>::T* __restrict__ prev, int store) {
    using St = Storage<S>;
    using T = typename St::T;
    constexpr int Q = L::kQ;
    if constexpr (sizeof(T) == 4) {
        constexpr int G = c2f_lanes<L, T>();
        if (i >= (long long)st.n_targets * G) return;
        const int t = (int)(i / G), part = (int)(i - (long long)t * G);
        const float4* __restrict__ g4 = static_cast<const float4*>(st.g) + part;  // row s: g4[s G]
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        auto add = [&](int2 e, const float4& v) {
            const float w = __int_as_float(e.y);
            acc[0] = acc[0] + w * v.x;
            acc[1] = acc[1] + w * v.y;
            acc[2] = acc[2] + w * v.z;
            acc[3] = acc[3] + w * v.w;
        };
        // rounds of four entries, predicated on the target's count; the next round's entries are
        // loaded beside this round's rows, so a round waits for one load, not two in a chain
        const int k1 = __ldg(st.offset + t + 1);
        int k = __ldg(st.offset + t);
        int2 en[4];
        auto entries = [&](int k0) {
#pragma unroll
            for (int e = 0; e < 4; ++e) en[e] = k0 + e < k1 ? __ldg(st.src_w32 + k0 + e) : make_int2(0, 0);
        };
        entries(k);
        for (; k < k1; k += 4) {
            int2 e4[4];
            float4 v4[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) e4[e] = en[e];
#pragma unroll
            for (int e = 0; e < 4; ++e)
                v4[e] = k + e < k1 ? __ldg(g4 + (long long)e4[e].x * G) : make_float4(0.f, 0.f, 0.f, 0.f);
            if (k + 4 < k1) entries(k + 4);
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if (k + e < k1) add(e4[e], v4[e]);
        }
        const Coord c = cell_coord(fgeo, st.target[t]);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int q = 4 * part + j;
            if (q >= Q) break;
            const long long iq = (long long)t * Q + q;
            float a = acc[j];
            if (save) save[iq] = a;
            if (!store) continue;
            if (prev) a = 0.5f * (prev[iq] + a);
            St::store(ff + post_stream_slot<L>(fgeo, c, q, f_even), a, fp);
        }
        return;
    }
    if (i >= (long long)st.n_targets * Q) return;
    const int t = (int)(i / Q), q = (int)(i - (long long)t * Q);
    const T* __restrict__ g = static_cast<const T*>(st.g);
    // entry k: its source row and weight (FP32 storages: one 8-byte load for both)
    auto entry = [&](int k, int& s, T& w) {
        if constexpr (sizeof(T) == 8) {
            s = __ldg(st.src + k);
            w = __ldg(st.weight + k);
        } else {
            const int2 e = __ldg(st.src_w32 + k);
            s = e.x;
            w = __int_as_float(e.y);
        }
    };
    T acc = (T)0;
    const int k1 = __ldg(st.offset + t + 1);
    int k = __ldg(st.offset + t);
    for (; k + 4 <= k1; k += 4) {
        int s4[4];
        T w4[4], g4[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) entry(k + e, s4[e], w4[e]);
#pragma unroll
        for (int e = 0; e < 4; ++e) g4[e] = __ldg(g + (long long)s4[e] * Q + q);
#pragma unroll
        for (int e = 0; e < 4; ++e) acc = acc + w4[e] * g4[e];
    }
    for (; k < k1; ++k) {
        int s;
        T w;
        entry(k, s, w);
        acc = acc + w * __ldg(g + (long long)s * Q + q);
    }
    if (save) save[i] = acc;
    if (!store) return;
    if (prev) acc = (T)0.5 * (prev[i] + acc);
    const Coord c = cell_coord(fgeo, st.target[t]);
    St::store(ff + post_stream_slot<L>(fgeo, c, q, f_even), acc, fp);
}

template <class L, class S>
__global__ void __launch_bounds__(kC2fThreads) c2f_kernel(S* __restrict__ ff, LevelGeom fgeo, int f_even,
                                                         StepParams fp, C2FStencil st,
                                                         typename Storage<S>::T* __restrict__ save,
                                                         const typename Storage<S>::T* __restrict__ prev, int store) {
    pdl_wait();
    pdl_trigger();
    c2f_thread<L, S>(blockIdx.x * (long long)blockDim.x + threadIdx.x, ff, fgeo, f_even, fp, st, save, prev, store);
}

// The coalescence nodes of a transfer: coarse cell, coincident fine cell, the fine level's saved
// macros and the relaxation-time ratio.
struct F2CJob {
    const int* coarse_cell;
    const int* fine_cell;
    int n;
    const double* fine_macro;
    double tau_ratio;
};

// Coalescence (TransferInfoToCoarseGrid, lbm_grid_interface.cpp:524-564): a coarse node of the
// inner coarse-to-fine layer takes rho, u of the coincident fine node (as stored by its last
// collision) and f = feq + tau_f2c (f_fine - feq) (NodeInfoFine2Coarse + PostStreamFine2Coarse,
// lbm_grid_interface.cpp:594-610, lbm_collision_models.cpp:259-267).
// One thread per (node, population q): a few thousand nodes give the launch Q times the threads,
// and each thread has one population load in flight with the node's macros; every thread of a node
// forms the same feq (the same operations in the same order) and keeps its q.
template <class L, class S>
__device__ __forceinline__ void f2c_thread(long long i, const S* __restrict__ ff, const LevelGeom& fgeo, int f_even,
                                           S* __restrict__ fc, const LevelGeom& cgeo, int c_even,
                                           const StepParams& fp, const StepParams& cp, const F2CJob& job) {
    using St = Storage<S>;
    constexpr int Q = L::kQ;
    if (i >= (long long)job.n * Q) return;
    const int t = (int)(i / Q), q = (int)(i - (long long)t * Q);
    const int fcell = job.fine_cell[t];
    const Coord cf = cell_coord(fgeo, fcell);
    const Coord cc = cell_coord(cgeo, job.coarse_cell[t]);
    const double* mac = job.fine_macro + (long long)fcell * 4;
    if constexpr (St::kDeviation) {
        const float v = St::load(ff + post_stream_slot<L>(fgeo, cf, q, f_even), fp);
        float deq[Q];
        feq_dev<L>((float)mac[0], (float)mac[1], (float)mac[2], (float)mac[3], deq);
        float e = deq[0];
#pragma unroll
        for (int k = 1; k < Q; ++k)
            if (k == q) e = deq[k];
        St::store(fc + post_stream_slot<L>(cgeo, cc, q, c_even), e + (float)job.tau_ratio * (v - e), cp);
    } else {
        const double v = St::load(ff + post_stream_slot<L>(fgeo, cf, q, f_even), fp);
        double feq[Q];
        feq_exact<L>(mac[0], mac[1], mac[2], mac[3], feq);
        double e = feq[0];
#pragma unroll
        for (int k = 1; k < Q; ++k)
            if (k == q) e = feq[k];
        St::store(fc + post_stream_slot<L>(cgeo, cc, q, c_even), e + job.tau_ratio * (v - e), cp);
    }
}

template <class L, class S>
__global__ void f2c_kernel(const S* __restrict__ ff, LevelGeom fgeo, int f_even, S* __restrict__ fc, LevelGeom cgeo,
                           int c_even, StepParams fp, StepParams cp, F2CJob job) {
    pdl_wait();
    pdl_trigger();
    f2c_thread<L, S>(blockIdx.x * (long long)blockDim.x + threadIdx.x, ff, fgeo, f_even, fc, cgeo, c_even, fp, cp, job);
}

// The explosion and the coalescence of one transfer in one launch: blocks [0, c2f_blocks) form the
// explosion targets, the others the coalescence nodes.  Used when no explosion target is a
// coalescence source: an explosion writes slot (t - c_q, opp q) or (t, q) of its target t, a
// coalescence reads the same slot of its fine node, so the two meet only where a target is that
// node, and running them side by side equals running them one after the other.
template <class L, class S>
__global__ void __launch_bounds__(kC2fThreads) c2f_f2c_kernel(S* __restrict__ ff, LevelGeom fgeo, int f_even,
                                                             StepParams fp, C2FStencil st,
                                                             typename Storage<S>::T* __restrict__ save, S* __restrict__ fc,
                                                             LevelGeom cgeo, int c_even, StepParams cp, F2CJob job,
                                                             unsigned c2f_blocks) {
    pdl_wait();
    pdl_trigger();
    if (blockIdx.x < c2f_blocks)
        c2f_thread<L, S>(blockIdx.x * (long long)blockDim.x + threadIdx.x, ff, fgeo, f_even, fp, st, save, nullptr, 1);
    else
        f2c_thread<L, S>((blockIdx.x - c2f_blocks) * (long long)blockDim.x + threadIdx.x, ff, fgeo, f_even, fc, cgeo,
                         c_even, fp, cp, job);
}

// ---------------------------------------------------------------- host exchange
template <class L, class S>
__global__ void scatter_kernel(S* __restrict__ f, LevelGeom geo, StepParams p, LevelMap m, int even_layout,
                               const uint64_t* __restrict__ codes, const double* __restrict__ fin, long long n,
                               int* __restrict__ bad) {
    using St = Storage<S>;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Coord c;
    bool folded = false;
    if (!code_to_node(codes[i], m, c, &folded)) {
        atomicExch(bad, 1);
        return;
    }
    // A periodic axis stores its duplicated maximum plane once, at coordinate 0.  Only the
    // minimum-plane code writes that node; the maximum-plane copy is ignored, so the result
    // does not depend on which of two disagreeing copies a thread happens to write last.
    if (folded) return;
    for (int q = 0; q < L::kQ; ++q) {
        double v = fin[i * L::kQ + q];
        if constexpr (St::kDeviation) v -= Tables<L>::w(q);
        St::store(f + post_stream_slot<L>(geo, c, q, even_layout), (typename St::T)v, p);
    }
}

template <class L, class S>
__global__ void gather_kernel(const S* __restrict__ f, LevelGeom geo, StepParams p, LevelMap m, int even_layout,
                              const uint64_t* __restrict__ codes, double* __restrict__ fout, double* __restrict__ rho_out,
                              double* __restrict__ u_out, long long n, int* __restrict__ bad) {
    using St = Storage<S>;
    using T = typename St::T;
    constexpr int Q = L::kQ;
    constexpr int D = L::kDims;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Coord c;
    if (!code_to_node(codes[i], m, c)) {
        atomicExch(bad, 1);
        return;
    }
    T v[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) v[q] = St::load(f + post_stream_slot<L>(geo, c, q, even_layout), p);
    if (fout) {
        for (int q = 0; q < Q; ++q) {
            double x = (double)v[q];
            if constexpr (St::kDeviation) x += Tables<L>::w(q);
            fout[i * Q + q] = x;
        }
    }
    if (rho_out) {
        // velocity recomputed from post-boundary f, as the reference's output does
        // (lbm_grid_interface.cpp:614-657), with the node's forces when the level is forced
        double F[3] = {0., 0., 0.};
        if (p.forced) {
            const long long self = (long long)(c.x[0] + geo.g[0]) +
                                   (long long)geo.a[0] * ((c.x[1] + geo.g[1]) + (long long)geo.a[1] * (c.x[2] + geo.g[2]));
            for (int a = 0; a < 3; ++a) F[a] = p.const_force[a] + (p.force ? p.force[self * 3 + a] : 0.);
        }
        if constexpr (St::kDeviation) {
            float rho, ux, uy, uz;
            macro_dev<L>(v, rho, ux, uy, uz);
            if (p.forced) {
                const float h = 0.5f * (float)p.dt / rho;
                ux += h * (float)F[0];
                uy += h * (float)F[1];
                uz += h * (float)F[2];
            }
            rho_out[i] = rho;
            u_out[i * D] = ux;
            u_out[i * D + 1] = uy;
            if (D == 3) u_out[i * D + 2] = uz;
        } else {
            double rho, ux, uy, uz;
            macro_exact<L>(v, rho, ux, uy, uz, p.forced ? F : nullptr, p.dt);
            rho_out[i] = rho;
            u_out[i * D] = ux;
            u_out[i * D + 1] = uy;
            if (D == 3) u_out[i * D + 2] = uz;
        }
    }
}

// ---------------------------------------------------------------- FP64 conservation sums
// Mass and momentum of every node of the level, accumulated in FP64: one partial per
// block into `partial`, then a single-block pass adds the partials in a fixed order
// (deterministic result for a given launch shape).
template <class L, class S>
__global__ void __launch_bounds__(256) conservation_partial_kernel(const S* __restrict__ f, LevelGeom geo,
                                                                   StepParams p, int even_layout,
                                                                   double* __restrict__ partial) {
    using St = Storage<S>;
    constexpr int Q = L::kQ;
    __shared__ double red[4][256 / 32];
    double acc[4] = {0., 0., 0., 0.};
    // blocks stride over the (y, z) rows of the box, threads over x: no per-node division
    const int rows = geo.n[1] * (L::kDims == 3 ? geo.n[2] : 1);
    for (int r = blockIdx.x; r < rows; r += gridDim.x) {
        Coord c;
        c.x[1] = r % geo.n[1];
        c.x[2] = L::kDims == 3 ? r / geo.n[1] : 0;
        for (int x = threadIdx.x; x < geo.n[0]; x += blockDim.x) {
            c.x[0] = x;
            if (geo.info) {
                const long long self = (long long)(c.x[0] + geo.g[0]) +
                                       (long long)geo.a[0] * ((c.x[1] + geo.g[1]) + (long long)geo.a[1] * (c.x[2] + geo.g[2]));
                if (!(__ldg(geo.info + self) & kInfoPresent)) continue;
            }
            double rho = 0., jx = 0., jy = 0., jz = 0.;
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                double v = (double)St::load(f + post_stream_slot<L>(geo, c, q, even_layout), p);
                if constexpr (St::kDeviation) v += Tables<L>::w(q);
                rho += v;
                if (Tables<L>::cx(q)) jx += Tables<L>::cx(q) > 0 ? v : -v;
                if (Tables<L>::cy(q)) jy += Tables<L>::cy(q) > 0 ? v : -v;
                if (L::kDims == 3 && Tables<L>::cz(q)) jz += Tables<L>::cz(q) > 0 ? v : -v;
            }
            acc[0] += rho;
            acc[1] += jx;
            acc[2] += jy;
            acc[3] += jz;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double v = acc[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0.;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
        partial[blockIdx.x * 4 + threadIdx.x] = v;
    }
}

__global__ void conservation_final_kernel(const double* __restrict__ partial, int nblocks, double* __restrict__ out);

}  // namespace zl
