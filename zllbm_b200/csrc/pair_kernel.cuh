// Two nodes per thread with packed FP32 pairs (fma.rn.f32x2 and friends, sm_100): the D3Q19 step
// of a full periodic box in deviation storage.  Thread t updates nodes x0 = 2t and x0 + 1 of a
// row.  Populations of the two nodes that sit side by side in a plane move as one 32-bit (FP16 /
// BF16) or 64-bit (FP32) access; the collision runs once on (node a, node b) pairs in the fused
// form of mrt_d3q19_fused, which halves its arithmetic instructions.  Same formulas as the
// scalar kernel; roundings can differ where the scalar build contracts a product and a sum into
// one FMA.  Requires an even row length (x0, x0 + 1 in one row, pair accesses aligned).
#pragma once
#include "aa_kernel.cuh"

namespace zl {

struct F2 {
    float2 v;
};
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return {__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return {__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 vfma(F2 a, F2 b, F2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ F2 splat(float s) { return {make_float2(s, s)}; }

// Two neighbouring slots of a plane as one access.
template <class S> struct PairIO;
template <> struct PairIO<float> {
    __device__ __forceinline__ static F2 load(const float* p) { return {__ldg(reinterpret_cast<const float2*>(p))}; }
    __device__ __forceinline__ static void store(float* p, F2 v) { *reinterpret_cast<float2*>(p) = v.v; }
    __device__ __forceinline__ static void store_sr(float* p, F2 v, uint32_t) { store(p, v); }
};
template <> struct PairIO<__half> {
    __device__ __forceinline__ static F2 load(const __half* p) {
        return {__half22float2(__ldg(reinterpret_cast<const __half2*>(p)))};
    }
    __device__ __forceinline__ static void store(__half* p, F2 v) {
        *reinterpret_cast<__half2*>(p) = __float22half2_rn(v.v);
    }
    __device__ __forceinline__ static void store_sr(__half* p, F2 v, uint32_t rbits) {
        *reinterpret_cast<uint32_t*>(p) = cvt_rs_f16x2(v.v.y, v.v.x, rbits);
    }
};
template <> struct PairIO<__nv_bfloat16> {
    __device__ __forceinline__ static F2 load(const __nv_bfloat16* p) {
        return {__bfloat1622float2(__ldg(reinterpret_cast<const __nv_bfloat162*>(p)))};
    }
    __device__ __forceinline__ static void store(__nv_bfloat16* p, F2 v) {
        *reinterpret_cast<__nv_bfloat162*>(p) = __float22bfloat162_rn(v.v);
    }
    __device__ __forceinline__ static void store_sr(__nv_bfloat16* p, F2 v, uint32_t rbits) {
        *reinterpret_cast<uint32_t*>(p) = cvt_rs_bf16x2(v.v.y, v.v.x, rbits);
    }
};

// mrt_d3q19_fused for node pairs (Mrt = false: SRT, every correction c_q is zero).
template <bool Mrt>
__device__ __forceinline__ void fused_pair(const F2* d, F2* out, const StepParams& p) {
    const float omega = p.omega32;
    const float* lam = p.mrt_coef;
    const F2 S1 = d[1] + d[2], D1 = d[1] - d[2];
    const F2 S2 = d[3] + d[4], D2 = d[3] - d[4];
    const F2 S3 = d[5] + d[6], D3 = d[5] - d[6];
    const F2 S4 = d[7] + d[10], D4 = d[7] - d[10];
    const F2 S5 = d[8] + d[9], D5 = d[8] - d[9];
    const F2 S6 = d[11] + d[14], D6 = d[11] - d[14];
    const F2 S7 = d[12] + d[13], D7 = d[12] - d[13];
    const F2 S8 = d[15] + d[18], D8 = d[15] - d[18];
    const F2 S9 = d[16] + d[17], D9 = d[16] - d[17];
    const F2 S23 = S2 + S3;
    const F2 Sa = S1 + S23;
    const F2 Sxy = S4 + S5, Sxz = S6 + S7, Syz = S8 + S9;
    const F2 Sd = (Sxy + Sxz) + Syz;
    const F2 drho = (d[0] + Sa) + Sd;
    const F2 X1 = D4 - D5, X2 = D6 - D7;
    const F2 Y1 = D4 + D5, Y2 = D8 - D9;
    const F2 Z1 = D6 + D7, Z2 = D8 + D9;
    const F2 X12 = X1 + X2, Y12 = Y1 + Y2, Z12 = Z1 + Z2;
    const F2 jx = D1 + X12, jy = D2 + Y12, jz = D3 + Z12;
    const F2 rho = vfma(drho, splat(p.inv_scale), splat(1.f));
    // inv_scale / rho through the fast reciprocal (two ulps; rho is close to 1)
    const F2 k = {make_float2(__fdividef(p.inv_scale, rho.v.x), __fdividef(p.inv_scale, rho.v.y))};
    const F2 ux = jx * k, uy = jy * k, uz = jz * k;
    const F2 ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
    const F2 usq = (ux2 + uy2) + uz2;
    const F2 G = splat(p.scale) * rho;
    const F2 Gu = G * usq;
    const F2 zero = splat(0.f);
    F2 c0 = zero, cx = zero, cy = zero, cz = zero, c_xy = zero, c_xz = zero, c_yz = zero;
    F2 a4x4 = zero, a6x4 = zero, a8x4 = zero, u1 = zero, u2 = zero, v1 = zero, v2 = zero, t1 = zero, t2 = zero;
    if constexpr (Mrt) {
        // relaxed moments of neq, times lambda_k = (s_k - omega) / |M_k|^2
        const F2 a1 = splat(19.f * lam[1]) * ((Sd - d[0]) - Gu);
        const F2 a2 = splat(lam[2]) * vfma(splat(5.5f), Gu, vfma(splat(9.f), d[0], vfma(splat(-7.f), Sa, splat(-2.f) * Sd)));
        const F2 a4 = splat(lam[4]) * vfma(splat(-10.f / 3.f), D1, splat(5.f / 3.f) * X12);
        const F2 a6 = splat(lam[6]) * vfma(splat(-10.f / 3.f), D2, splat(5.f / 3.f) * Y12);
        const F2 a8 = splat(lam[8]) * vfma(splat(-10.f / 3.f), D3, splat(5.f / 3.f) * Z12);
        const F2 hG = splat(0.5f) * G;
        const F2 a10 = splat(lam[10]) * vfma(hG, vfma(splat(3.f), ux2, zero - usq),
                                             vfma(splat(-4.f), S1, vfma(splat(2.f), S23, (Sxy + Sxz) - splat(2.f) * Syz)));
        const F2 a12 = splat(lam[12]) * vfma(hG, uy2 - uz2, vfma(splat(2.f), S3 - S2, Sxy - Sxz));
        const F2 a16 = splat(lam[16]) * (X1 - X2), a17 = splat(lam[17]) * (Y2 - Y1), a18 = splat(lam[18]) * (Z1 - Z2);
        const F2 e_ax = vfma(splat(-11.f), a1, splat(-4.f) * a2);
        const F2 e_dg = vfma(splat(8.f), a1, a2);
        c0 = vfma(splat(-30.f), a1, splat(12.f) * a2);
        cx = vfma(splat(-4.f), a10, e_ax);
        cy = vfma(splat(2.f), a10 - a12, e_ax);
        cz = vfma(splat(2.f), a10 + a12, e_ax);
        c_xy = e_dg + (a10 + a12);
        c_xz = e_dg + (a10 - a12);
        c_yz = vfma(splat(-2.f), a10, e_dg);
        a4x4 = splat(4.f) * a4;
        a6x4 = splat(4.f) * a6;
        a8x4 = splat(4.f) * a8;
        u1 = a4 + a16;  // q7: u1 + u2, q8: u2 - u1
        u2 = a6 - a17;
        v1 = a4 - a16;  // q11: v1 + v2, q12: v2 - v1
        v2 = a8 + a18;
        t1 = a6 + a17;  // q15: t1 + t2, q16: t2 - t1
        t2 = a8 - a18;
    }
    // omega feq: w (B + 4.5 G (c.u)^2) even, 3 w (c.j) odd, B = drho - 1.5 G u^2
    const F2 B = vfma(splat(-1.5f), Gu, drho);
    const float ow0 = omega * (1.f / 3.f), ow1 = omega * (1.f / 18.f), ow2 = omega * (1.f / 36.f);
    const F2 K1 = splat(4.5f * ow1) * G, L1 = splat(ow1) * B;
    const F2 K2 = splat(4.5f * ow2) * G, L2 = splat(ow2) * B, K2x2 = K2 + K2;
    const F2 o1 = splat(ow1 * 3.f), o2 = splat(ow2 * 3.f);
    // (1 - omega) d_q of a pair of opposite directions from their sum and difference
    const F2 h = splat(0.5f * (1.f - omega));
    out[0] = vfma(splat(1.f - omega), d[0], vfma(splat(ow0), B, zero - c0));
    auto pair = [&](int q, int o, F2 S, F2 D, F2 A, F2 Bo) {
        const F2 e = vfma(h, S, A), od = vfma(h, D, Bo);
        out[q] = e + od;
        out[o] = e - od;
    };
    pair(1, 2, S1, D1, vfma(K1, ux2, L1) - cx, vfma(o1, jx, a4x4));
    pair(3, 4, S2, D2, vfma(K1, uy2, L1) - cy, vfma(o1, jy, a6x4));
    pair(5, 6, S3, D3, vfma(K1, uz2, L1) - cz, vfma(o1, jz, a8x4));
    {
        const F2 P = vfma(K2, ux2 + uy2, L2) - c_xy, Q = K2x2 * (ux * uy);
        pair(7, 10, S4, D4, P + Q, vfma(o2, jx + jy, zero - (u1 + u2)));
        pair(8, 9, S5, D5, P - Q, vfma(o2, jy - jx, u1 - u2));
    }
    {
        const F2 P = vfma(K2, ux2 + uz2, L2) - c_xz, Q = K2x2 * (ux * uz);
        pair(11, 14, S6, D6, P + Q, vfma(o2, jx + jz, zero - (v1 + v2)));
        pair(12, 13, S7, D7, P - Q, vfma(o2, jz - jx, v1 - v2));
    }
    {
        const F2 P = vfma(K2, uy2 + uz2, L2) - c_yz, Q = K2x2 * (uy * uz);
        pair(15, 18, S8, D8, P + Q, vfma(o2, jy + jz, zero - (t1 + t2)));
        pair(16, 17, S9, D9, P - Q, vfma(o2, jz - jy, t1 - t2));
    }
}

// Nodes x0 and x0 + 1 of a row of a full periodic box (or a slab of one, geo.ring: z neighbours
// in the ghost planes) with an even row length.  Rows whose y or z neighbours wrap take the scalar
// node update twice.
template <class S, int Coll, bool Odd>
__global__ void __launch_bounds__(256, 2) aa_pair_kernel(S* __restrict__ f, LevelGeom geo, StepParams p) {
    pdl_wait();
    pdl_trigger();
    using Tb = Tables<D3Q19>;
    using St = Storage<S>;
    using IO = PairIO<S>;
    const int x0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z + geo.z0;
    if (sizeof(S) == 2 && (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0)
        sr_advance(p, Odd, sr_seed(p, Odd), true);
    if (x0 >= geo.n[0] || y >= geo.n[1]) return;
    const int gz = geo.g[2];  // 1 on a slab: z rows never wrap
    if (!(y > 0 && y < geo.n[1] - 1 && (gz || (z > 0 && z < geo.n[2] - 1)))) {
        Coord c;
        c.x[0] = x0;
        c.x[1] = y;
        c.x[2] = z;
        aa_node<D3Q19, S, Coll, Odd, false, false, 0>(f, geo, p, c);
        c.x[0] = x0 + 1;
        aa_node<D3Q19, S, Coll, Odd, false, false, 0>(f, geo, p, c);
        return;
    }
    const int n0 = geo.n[0];
    const int row = geo.a[0] * (y + geo.a[1] * (z + gz));
    // columns x0 - 1, x0, x0 + 1, x0 + 2 of the row (x wrapped)
    S* const pc[4] = {f + (row + (x0 == 0 ? n0 - 1 : x0 - 1)), f + (row + x0), f + (row + x0 + 1),
                      f + (row + (x0 + 2 == n0 ? 0 : x0 + 2))};
    const long long st = geo.stride;
    const int a0 = geo.a[0], a01 = geo.a[0] * geo.a[1];
    auto off = [&](int q, int dy, int dz) -> long long { return q * st + (long long)(dy * a0 + dz * a01); };
    F2 pre[19], post[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (!Odd || q == 0) {
            pre[q] = IO::load(pc[1] + off(q, 0, 0));
        } else if (Tb::cx(q) == 0) {
            pre[q] = IO::load(pc[1] + off(Tb::opp(q), -Tb::cy(q), -Tb::cz(q)));
        } else {
            const long long o = off(Tb::opp(q), -Tb::cy(q), -Tb::cz(q));
            pre[q] = {make_float2(St::load_raw(pc[1 - Tb::cx(q)] + o), St::load_raw(pc[2 - Tb::cx(q)] + o))};
        }
    }
    fused_pair<Coll == kMrt>(pre, post, p);
    if (sizeof(S) == 2 && p.sr_seed) {
        // stochastic rounding of the 16-bit stores, one random stream per node pair
        SrBits rng(sr_seed(p, Odd), (uint32_t)((row + x0) >> 1));
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const uint32_t r = rng.next();
            if (!Odd || q == 0) {
                IO::store_sr(pc[1] + off(Tb::opp(q), 0, 0), post[q], r);
            } else if (Tb::cx(q) == 0) {
                IO::store_sr(pc[1] + off(q, Tb::cy(q), Tb::cz(q)), post[q], r);
            } else {
                const long long o = off(q, Tb::cy(q), Tb::cz(q));
                St::store_raw_sr(pc[1 + Tb::cx(q)] + o, post[q].v.x, r);
                St::store_raw_sr(pc[2 + Tb::cx(q)] + o, post[q].v.y, r ^ 0x9e3779b9u);
            }
        }
        return;
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (!Odd || q == 0) {
            IO::store(pc[1] + off(Tb::opp(q), 0, 0), post[q]);
        } else if (Tb::cx(q) == 0) {
            IO::store(pc[1] + off(q, Tb::cy(q), Tb::cz(q)), post[q]);
        } else {
            const long long o = off(q, Tb::cy(q), Tb::cz(q));
            St::store_raw(pc[1 + Tb::cx(q)] + o, post[q].v.x);
            St::store_raw(pc[2 + Tb::cx(q)] + o, post[q].v.y);
        }
    }
}

}  // namespace zl
