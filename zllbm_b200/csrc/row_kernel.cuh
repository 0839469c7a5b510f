// One warp per x-row: the D3Q19 step of a full periodic box in 16-bit deviation storage (FP16 /
// BF16) whose rows hold 32 V nodes (V = 8: 256, V = 4: 128).  Lane l owns nodes 8l .. 8l + 7
// (V = 8) of its row and moves each population plane as one 128-bit (V = 8) or 64-bit (V = 4)
// access.  The AA pattern's odd step shifts the c_x != 0 directions by one node along x; the
// warp covers the whole periodic row, so the shifted vector is the lane's own vector
// funnel-shifted by 16 bits with one element from the neighbouring lane (one warp shuffle, the
// row's wrap-around being lane 31 <-> lane 0).  Row offsets of the nine neighbouring rows are
// computed once per lane (y / z wrap-around included).  The collision is the packed-pair form of
// aa_pair_kernel (fused_pair) on nodes (2k, 2k + 1) of the lane's vector, so both kernels round
// identically.
#pragma once
#include <type_traits>
#include "pair_kernel.cuh"

namespace zl {

// Block x of LevelGeom::block that selects the row kernel; block y is then the rows (warps) per block.
constexpr int kRowKernelBlockX = 1 << 20;

template <class S> struct HalfPairIO;
template <> struct HalfPairIO<__half> {
    __device__ __forceinline__ static F2 unpack(uint32_t w) {
        __half2 h;
        memcpy(&h, &w, 4);
        return {__half22float2(h)};
    }
    __device__ __forceinline__ static uint32_t pack(F2 v) {
        const __half2 h = __float22half2_rn(v.v);
        uint32_t w;
        memcpy(&w, &h, 4);
        return w;
    }
    __device__ __forceinline__ static uint32_t pack_sr(F2 v, uint32_t rbits) { return cvt_rs_f16x2(v.v.y, v.v.x, rbits); }
};
template <> struct HalfPairIO<__nv_bfloat16> {
    __device__ __forceinline__ static F2 unpack(uint32_t w) {
        __nv_bfloat162 h;
        memcpy(&h, &w, 4);
        return {__bfloat1622float2(h)};
    }
    __device__ __forceinline__ static uint32_t pack(F2 v) {
        const __nv_bfloat162 h = __float22bfloat162_rn(v.v);
        uint32_t w;
        memcpy(&w, &h, 4);
        return w;
    }
    __device__ __forceinline__ static uint32_t pack_sr(F2 v, uint32_t rbits) { return cvt_rs_bf16x2(v.v.y, v.v.x, rbits); }
};

// V 16-bit values of one plane as V / 2 32-bit words (element 2k in the low half of word k).
template <int V> struct RowVec {
    uint32_t w[V / 2];
};

template <int V>
__device__ __forceinline__ RowVec<V> row_load(const void* p) {
    RowVec<V> r;
    if constexpr (V == 8) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
        r.w[0] = v.x; r.w[1] = v.y; r.w[2] = v.z; r.w[3] = v.w;
    } else {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
        r.w[0] = v.x; r.w[1] = v.y;
    }
    return r;
}

template <int V>
__device__ __forceinline__ void row_store(void* p, const RowVec<V>& r) {
    if constexpr (V == 8) {
        *reinterpret_cast<uint4*>(p) = make_uint4(r.w[0], r.w[1], r.w[2], r.w[3]);
    } else {
        *reinterpret_cast<uint2*>(p) = make_uint2(r.w[0], r.w[1]);
    }
}

// out[i] = in[i - 1] with out[0] = last element of the previous lane (row wrap-around at lane 0).
template <int V>
__device__ __forceinline__ RowVec<V> row_shift_up(const RowVec<V>& in, int lane) {
    constexpr int K = V / 2;
    const uint32_t prev = __shfl_sync(0xffffffffu, in.w[K - 1], (lane + 31) & 31);
    RowVec<V> out;
#pragma unroll
    for (int k = K - 1; k > 0; --k) out.w[k] = __funnelshift_l(in.w[k - 1], in.w[k], 16);
    out.w[0] = __funnelshift_l(prev, in.w[0], 16);
    return out;
}

// out[i] = in[i + 1] with out[V - 1] = first element of the next lane (wrap-around at lane 31).
template <int V>
__device__ __forceinline__ RowVec<V> row_shift_down(const RowVec<V>& in, int lane) {
    constexpr int K = V / 2;
    const uint32_t next = __shfl_sync(0xffffffffu, in.w[0], (lane + 1) & 31);
    RowVec<V> out;
#pragma unroll
    for (int k = 0; k < K - 1; ++k) out.w[k] = __funnelshift_r(in.w[k], in.w[k + 1], 16);
    out.w[K - 1] = __funnelshift_r(in.w[K - 1], next, 16);
    return out;
}

template <class S, int Coll, bool Odd, int V>
__global__ void __launch_bounds__(128, 3) aa_row_kernel(S* __restrict__ f, LevelGeom geo, StepParams p) {
    pdl_wait();
    pdl_trigger();
    static_assert(sizeof(S) == 2 && (V == 4 || V == 8), "16-bit storage, 4 or 8 nodes per lane");
    using Tb = Tables<D3Q19>;
    using IO = HalfPairIO<S>;
    constexpr int K = V / 2;
    const int lane = threadIdx.x & 31;
    const int y = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int z = blockIdx.y + geo.z0;
    if ((blockIdx.x | blockIdx.y | threadIdx.x) == 0) sr_advance(p, Odd, sr_seed(p, Odd), true);
    if (y >= geo.n[1]) return;  // whole warp: every shuffle below has all 32 lanes
    const int n1 = geo.n[1], n2 = geo.n[2];
    // element offsets of the rows (y + dy, z + dz), wrapped (z: through the ghost planes of a
    // slab, geo.ring, box coordinate z + 1), plus this lane's first node
    const int ym = y == 0 ? n1 - 1 : y - 1, yp = y == n1 - 1 ? 0 : y + 1;
    const int gz = geo.g[2];
    const int zc = z + gz;
    const int zm = gz ? z : (z == 0 ? n2 - 1 : z - 1), zp = gz ? z + 2 : (z == n2 - 1 ? 0 : z + 1);
    const uint32_t a0 = (uint32_t)geo.a[0], a1 = (uint32_t)geo.a[1];
    const uint32_t x0 = (uint32_t)(lane * V);
    auto rowoff = [&](int dy, int dz) -> uint32_t {
        const int yy = dy < 0 ? ym : (dy > 0 ? yp : y);
        const int zz = dz < 0 ? zm : (dz > 0 ? zp : zc);
        return a0 * ((uint32_t)yy + a1 * (uint32_t)zz) + x0;
    };
    const long long st = geo.stride;
    auto at = [&](int q, uint32_t off) -> S* { return f + (q * st + off); };

    RowVec<V> v[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (!Odd || q == 0) {
            v[q] = row_load<V>(at(q, rowoff(0, 0)));
        } else {
            // f(x, q) of the odd step sits in slot (x - c_q, opp q)
            const RowVec<V> r = row_load<V>(at(Tb::opp(q), rowoff(-Tb::cy(q), -Tb::cz(q))));
            if (Tb::cx(q) == 1) v[q] = row_shift_up<V>(r, lane);
            else if (Tb::cx(q) == -1) v[q] = row_shift_down<V>(r, lane);
            else v[q] = r;
        }
    }
    // stochastic rounding (p.sr_seed): one random stream per lane
    const bool sr = p.sr_seed != nullptr;
    SrBits rng(sr ? sr_seed(p, Odd) : 0u, (uint32_t)((geo.n[1] * z + y) * 32 + lane));
#pragma unroll
    for (int k = 0; k < K; ++k) {
        F2 pre[19], post[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) pre[q] = IO::unpack(v[q].w[k]);
        fused_pair<Coll == kMrt>(pre, post, p);
        if (sr) {
#pragma unroll
            for (int q = 0; q < 19; ++q) v[q].w[k] = IO::pack_sr(post[q], rng.next());
        } else {
#pragma unroll
            for (int q = 0; q < 19; ++q) v[q].w[k] = IO::pack(post[q]);
        }
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (!Odd || q == 0) {
            row_store<V>(at(Tb::opp(q), rowoff(0, 0)), v[q]);
        } else {
            // post-collision f(x, q) goes to slot (x + c_q, q)
            S* dst = at(q, rowoff(Tb::cy(q), Tb::cz(q)));
            if (Tb::cx(q) == 1) row_store<V>(dst, row_shift_up<V>(v[q], lane));
            else if (Tb::cx(q) == -1) row_store<V>(dst, row_shift_down<V>(v[q], lane));
            else row_store<V>(dst, v[q]);
        }
    }
}

// Full periodic D3Q19 box (no ghost frame), or a slab of one (geo.ring: ghost planes in z only), in
// 16-bit storage whose rows are 32 V nodes long and whose plane stride keeps every lane's vector
// aligned.
inline int row_kernel_width(const LevelGeom& geo) {
    if (!geo.periodic[0] || !geo.periodic[1] || !(geo.periodic[2] || geo.ring)) return 0;
    if (geo.g[0] || geo.g[1] || geo.g[2] != (geo.ring ? 1 : 0) || geo.a[0] != geo.n[0] || geo.a[1] != geo.n[1]) return 0;
    const int v = geo.n[0] / 32;
    if (geo.n[0] != 32 * v || (v != 4 && v != 8)) return 0;
    if (geo.stride % 8) return 0;
    return v;
}

}  // namespace zl
