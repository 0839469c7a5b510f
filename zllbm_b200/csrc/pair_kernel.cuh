// Two nodes per thread with packed FP32 pairs (fma.rn.f32x2 and friends, sm_100): the
// D3Q19 step of a full periodic box in deviation storage.  Thread t updates nodes 2t and 2t + 1
// of a row; the collision runs once on (node a, node b) pairs, which halves its arithmetic
// instructions.  Same formulas as the scalar kernel; roundings can differ where the scalar
// build contracts a product and a sum into one FMA.
#pragma once
#include "aa_kernel.cuh"

namespace zl {

struct F2 {
    float2 v;
};
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return {__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)}; }
__device__ __forceinline__ F2 operator-(F2 a) { return {make_float2(-a.v.x, -a.v.y)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return {__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(float s, F2 b) { return {__fmul2_rn(make_float2(s, s), b.v)}; }
__device__ __forceinline__ F2 operator/(F2 a, F2 b) { return {make_float2(a.v.x / b.v.x, a.v.y / b.v.y)}; }
__device__ __forceinline__ F2 vfma(F2 a, F2 b, F2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ F2 splat(float s) { return {make_float2(s, s)}; }

// The factored D3Q19 MRT collision (mrt_d3q19_dev) for node pairs.
template <class V>
__device__ __forceinline__ void mrt_d3q19_v(const V* d, const V* n, V* out, V omega, const float* lam) {
    // pair sums / differences over opposite directions
    const V S1 = n[1] + n[2], D1 = n[1] - n[2];
    const V S2 = n[3] + n[4], D2 = n[3] - n[4];
    const V S3 = n[5] + n[6], D3 = n[5] - n[6];
    const V S4 = n[7] + n[10], D4 = n[7] - n[10];
    const V S5 = n[8] + n[9], D5 = n[8] - n[9];
    const V S6 = n[11] + n[14], D6 = n[11] - n[14];
    const V S7 = n[12] + n[13], D7 = n[12] - n[13];
    const V S8 = n[15] + n[18], D8 = n[15] - n[18];
    const V S9 = n[16] + n[17], D9 = n[16] - n[17];
    const V Sa = S1 + S2 + S3;
    const V Sxy = S4 + S5, Sxz = S6 + S7, Syz = S8 + S9;
    const V Sd = Sxy + Sxz + Syz;
    const V m1 = -30.f * n[0] - 11.f * Sa + 8.f * Sd;
    const V m2 = 12.f * n[0] - 4.f * Sa + Sd;
    const V m10 = -4.f * S1 + 2.f * (S2 + S3) + Sxy + Sxz - 2.f * Syz;
    const V m12 = -2.f * S2 + 2.f * S3 + Sxy - Sxz;
    const V X1 = D4 - D5, X2 = D6 - D7;
    const V Y1 = D4 + D5, Y2 = D8 - D9;
    const V Z1 = D6 + D7, Z2 = D8 + D9;
    const V m4 = -4.f * D1 + X1 + X2, m16 = X1 - X2;
    const V m6 = -4.f * D2 + Y1 + Y2, m17 = -Y1 + Y2;
    const V m8 = -4.f * D3 + Z1 + Z2, m18 = Z1 - Z2;
    // lambda_k = (s_k - omega) / |M_k|^2
    const V a1 = lam[1] * m1, a2 = lam[2] * m2;
    const V a4 = lam[4] * m4, a6 = lam[6] * m6, a8 = lam[8] * m8;
    const V a10 = lam[10] * m10, a12 = lam[12] * m12;
    const V a16 = lam[16] * m16, a17 = lam[17] * m17, a18 = lam[18] * m18;
    const V e_ax = -11.f * a1 - 4.f * a2;
    const V e_dg = 8.f * a1 + a2;
    V c[19];
    c[0] = -30.f * a1 + 12.f * a2;
    {
        const V E = e_ax - 4.f * a10, O = -4.f * a4;
        c[1] = E + O; c[2] = E - O;
    }
    {
        const V E = e_ax + 2.f * a10 - 2.f * a12, O = -4.f * a6;
        c[3] = E + O; c[4] = E - O;
    }
    {
        const V E = e_ax + 2.f * a10 + 2.f * a12, O = -4.f * a8;
        c[5] = E + O; c[6] = E - O;
    }
    const V e_xy = e_dg + a10 + a12, e_xz = e_dg + a10 - a12, e_yz = e_dg - 2.f * a10;
    {
        const V O = a4 + a6 + a16 - a17;   // q = 7 (+1,+1,0), opposite 10
        c[7] = e_xy + O; c[10] = e_xy - O;
    }
    {
        const V O = -a4 + a6 - a16 - a17;  // q = 8 (-1,+1,0), opposite 9
        c[8] = e_xy + O; c[9] = e_xy - O;
    }
    {
        const V O = a4 + a8 - a16 + a18;   // q = 11 (+1,0,+1), opposite 14
        c[11] = e_xz + O; c[14] = e_xz - O;
    }
    {
        const V O = -a4 + a8 + a16 + a18;  // q = 12 (-1,0,+1), opposite 13
        c[12] = e_xz + O; c[13] = e_xz - O;
    }
    {
        const V O = a6 + a8 + a17 - a18;   // q = 15 (0,+1,+1), opposite 18
        c[15] = e_yz + O; c[18] = e_yz - O;
    }
    {
        const V O = -a6 + a8 - a17 - a18;  // q = 16 (0,-1,+1), opposite 17
        c[16] = e_yz + O; c[17] = e_yz - O;
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) out[q] = vfma(-omega, n[q], d[q]) - c[q];
}


// feq_neq_dev for a pair of nodes (no forcing): d are deviations times `scale`.
__device__ __forceinline__ void feq_neq_pair(const F2* d, F2* neq, float scale, float inv_scale) {
    using Tb = Tables<D3Q19>;
    F2 drho = d[0], jx = splat(0.f), jy = splat(0.f), jz = splat(0.f);
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        drho = drho + d[q];
        if (Tb::cx(q)) jx = Tb::cx(q) == 1 ? jx + d[q] : jx - d[q];
        if (Tb::cy(q)) jy = Tb::cy(q) == 1 ? jy + d[q] : jy - d[q];
        if (Tb::cz(q)) jz = Tb::cz(q) == 1 ? jz + d[q] : jz - d[q];
    }
    const F2 rho = vfma(drho, splat(inv_scale), splat(1.f));
    const F2 k = splat(inv_scale) / rho;
    const F2 ux = jx * k, uy = jy * k, uz = jz * k;
    const F2 usq15 = 1.5f * vfma(ux, ux, vfma(uy, uy, uz * uz));
    const F2 srho = scale * rho;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const int opp = Tb::opp(q);
        if (opp < q) continue;
        F2 cu = splat(0.f);
        if (Tb::cx(q)) cu = Tb::cx(q) > 0 ? cu + ux : cu - ux;
        if (Tb::cy(q)) cu = Tb::cy(q) > 0 ? cu + uy : cu - uy;
        if (Tb::cz(q)) cu = Tb::cz(q) > 0 ? cu + uz : cu - uz;
        const float w = (float)Tb::w(q);
        const F2 even = w * vfma(srho, vfma(4.5f * cu, cu, -usq15), drho);
        if (q == 0) {
            neq[0] = d[0] - even;
        } else {
            const F2 odd = (3.f * w) * (srho * cu);
            neq[q] = d[q] - (even + odd);
            neq[opp] = d[opp] - (even - odd);
        }
    }
}

template <class S, int Coll, bool Odd>
__global__ void __launch_bounds__(256, 2) aa_pair_kernel(S* __restrict__ f, LevelGeom geo, StepParams p) {
    using Tb = Tables<D3Q19>;
    using St = Storage<S>;
    const int x0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
    if (x0 >= geo.n[0] || y >= geo.n[1]) return;
    const bool second = x0 + 1 < geo.n[0];
    // box columns x0 - 1 .. x0 + 2 (periodic wrap), rows of y, z +- 1
    int bx[4], row[3][3];
    {
        int by[3], bz[3];
#pragma unroll
        for (int d = -1; d <= 2; ++d) bx[d + 1] = wrap_or_ghost(x0 + d, geo.n[0], 0, 1);
#pragma unroll
        for (int d = -1; d <= 1; ++d) {
            by[d + 1] = wrap_or_ghost(y + d, geo.n[1], 0, 1);
            bz[d + 1] = wrap_or_ghost(z + d, geo.n[2], 0, 1);
        }
#pragma unroll
        for (int dy = 0; dy < 3; ++dy)
#pragma unroll
            for (int dz = 0; dz < 3; ++dz) row[dy][dz] = geo.a[0] * (by[dy] + geo.a[1] * bz[dz]);
    }
    // node a at column 1 of bx, node b at column 2
    auto cell = [&](int node, int dx, int dy, int dz) -> int { return bx[1 + node + dx] + row[dy + 1][dz + 1]; };
    const long long st = geo.stride;
    F2 pre[19], neq[19], post[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        float a, b;
        if (Odd && q != 0) {
            const S* pl = f + Tb::opp(q) * st;
            a = St::load_raw(pl + cell(0, -Tb::cx(q), -Tb::cy(q), -Tb::cz(q)));
            b = second ? St::load_raw(pl + cell(1, -Tb::cx(q), -Tb::cy(q), -Tb::cz(q))) : a;
        } else {
            const S* pl = f + q * st;
            a = St::load_raw(pl + cell(0, 0, 0, 0));
            b = second ? St::load_raw(pl + cell(1, 0, 0, 0)) : a;
        }
        pre[q] = {make_float2(a, b)};
    }
    feq_neq_pair(pre, neq, p.scale, p.inv_scale);
    const F2 omega = splat(p.omega32);
    if (Coll == kSrt) {
#pragma unroll
        for (int q = 0; q < 19; ++q) post[q] = vfma(-omega, neq[q], pre[q]);
    } else {
        mrt_d3q19_v<F2>(pre, neq, post, omega, p.mrt_coef);
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (Odd && q != 0) {
            S* pl = f + q * st;
            St::store_raw(pl + cell(0, Tb::cx(q), Tb::cy(q), Tb::cz(q)), post[q].v.x);
            if (second) St::store_raw(pl + cell(1, Tb::cx(q), Tb::cy(q), Tb::cz(q)), post[q].v.y);
        } else {
            S* pl = f + Tb::opp(q) * st;
            St::store_raw(pl + cell(0, 0, 0, 0), post[q].v.x);
            if (second) St::store_raw(pl + cell(1, 0, 0, 0), post[q].v.y);
        }
    }
}

}  // namespace zl
