// Learned LES closure: node features, the 24 -> 64 -> 64 -> 1 network on tcgen05 tensor cores,
// and the shared-memory tile layout its kernels use.
//
// The closure has no counterpart in the reference, which hard-wires Smagorinsky
// (lbm_project/les_models/lbm_les_smagorinsky.cpp:22-94).  It keeps that model's relaxation
// formula and replaces the constant: C = 18 c with c = 0.01 clamp(y, 0, 8) from the network, so
// y = 1 is Smagorinsky with Cs = 0.1 and a network that is not set (or a non-finite y) falls
// back to the configured Smagorinsky constant.
//
// Layers: Z1 = W1 x_hat + b1, A1 = gelu(Z1), Z2 = W2 A1 + b2, A2 = gelu(Z2), y = w3 . A2 + b3, with
// x_hat = (x - mean) * inv_std and gelu the tanh form 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))).
// x_hat, W1, A1, W2 (and in training dZ2, dZ1) are BF16 tensor-core operands; everything else is FP32.
#pragma once
#include "aa_kernel.cuh"
#include "tc.cuh"

namespace zl {
namespace closure {

constexpr int kIn = 24, kHid = 64, kTile = 128;
// offsets in the flat parameter array (the zl_mlp struct)
constexpr int oW1 = 0, oB1 = oW1 + kHid * kIn, oW2 = oB1 + kHid, oB2 = oW2 + kHid * kHid, oW3 = oB2 + kHid,
              oB3 = oW3 + kHid, oMean = oB3 + 1, oInvStd = oMean + kIn, kFlat = oInvStd + kIn;
constexpr int kTrainable = oMean;
static_assert(kTrainable == 5825, "parameter count");

constexpr float kGeluK = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float kGeluA = 0.044715f;
constexpr float kCUnit = 0.01f;
constexpr float kYMax = 8.f;
constexpr uint32_t kWaitLimit = 1u << 22;  // mbarrier polls before a wait gives up

// ---------------------------------------------------------------- tiles (bytes, no swizzle)
// X  [128 samples x 32]: x_hat (24), a ones column (24), zeros        row groups 512 B apart
// A1 [128 samples x 80]: A1 (64), a ones column (64), zeros           1280 B
// DZ [128 samples x 128]: dZ (64), zeros (the M = 128 padding of the weight-gradient products)
// W1 [64 x 32]: W1 (24), b1 (24), zeros;  W2 [64 x 80]: W2 (64), b2 (64), zeros
// The ones columns carry the biases through the products: Z1 = [X | 1] [W1 | b1]^T, likewise Z2.
constexpr uint32_t kSboX = 512, kSboA1 = 1280, kSboDz = 2048, kSboW1 = 512, kSboW2 = 1280;
constexpr uint32_t kBytesX = 128 * kSboX / 8, kBytesA1 = 128 * kSboA1 / 8, kBytesDz = 128 * kSboDz / 8,
                   kBytesW1 = 64 * kSboW1 / 8, kBytesW2 = 64 * kSboW2 / 8;
// every descriptor stays inside its buffer
static_assert(tc::extent_kmajor(128, kSboX, 2) <= kBytesX, "X as A (K = 32)");
static_assert(tc::extent_mnmajor(32, kSboX, 8) <= kBytesX, "X as B of dW1 (N = 32, K = 128)");
static_assert(tc::extent_kmajor(128, kSboA1, 5) <= kBytesA1, "[A1 | 1] as A (K = 80)");
static_assert(tc::extent_mnmajor(80, kSboA1, 8) <= kBytesA1, "A1 as B of dW2 (N = 80, K = 128)");
static_assert(tc::extent_kmajor(128, kSboDz, 4) <= kBytesDz, "dZ2 as A of dA1 (K = 64)");
static_assert(tc::extent_mnmajor(128, kSboDz, 8) <= kBytesDz, "dZ as A of dW (M = 128, K = 128)");
static_assert(tc::extent_kmajor(64, kSboW1, 2) <= kBytesW1, "W1 as B (N = 64, K = 32)");
static_assert(tc::extent_kmajor(64, kSboW2, 5) <= kBytesW2, "[W2 | b2] as B (N = 64, K = 80)");
static_assert(tc::extent_mnmajor(64, kSboW2, 4) <= kBytesW2, "W2^T as B of dA1 (N = 64, K = 64)");

constexpr uint32_t kIdescFwd = tc::idesc_bf16(128, 64, false, false);   // X W1^T, A1 W2^T
constexpr uint32_t kIdescDa1 = tc::idesc_bf16(128, 64, false, true);    // dZ2 W2
constexpr uint32_t kIdescDw2 = tc::idesc_bf16(128, 80, true, true);     // dZ2^T [A1 | 1]
constexpr uint32_t kIdescDw1 = tc::idesc_bf16(128, 32, true, true);     // dZ1^T [X | 1]

__device__ __forceinline__ float gelu(float z, float& t) {
    t = tanhf(kGeluK * fmaf(kGeluA * z, z * z, z));
    return 0.5f * z * (1.f + t);
}
// Inference: the same GELU on packed BF16 pairs (the result is a BF16 operand anyway):
// z^2, 1 + a z^2, k z, k z (1 + a z^2), tanh.approx.bf16x2, z/2, z/2 + z/2 t -- every step rounds to
// BF16 (constants a, k rounded to BF16 too).
// The constants are BF16 bit patterns (a = 0x3d37, k = 0x3f4c, 1 = 0x3f80, 1/2 = 0x3f00, each in
// both halves), so that no conversion runs per call.
__device__ __forceinline__ __nv_bfloat162 bf16x2_bits(uint32_t b) {
    __nv_bfloat162 v;
    memcpy(&v, &b, 4);
    return v;
}
__device__ __forceinline__ uint32_t gelu_bf16x2(float z0, float z1) {
    const __nv_bfloat162 z = __floats2bfloat162_rn(z0, z1);
    const __nv_bfloat162 a = bf16x2_bits(0x3d373d37u), k = bf16x2_bits(0x3f4c3f4cu), one = bf16x2_bits(0x3f803f80u),
                         half = bf16x2_bits(0x3f003f00u);
    const __nv_bfloat162 p = __hfma2(__hmul2(z, z), a, one);
    const __nv_bfloat162 arg = __hmul2(__hmul2(z, k), p);
    uint32_t t;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(*reinterpret_cast<const uint32_t*>(&arg)));
    const __nv_bfloat162 hz = __hmul2(z, half);
    const __nv_bfloat162 out = __hfma2(hz, *reinterpret_cast<const __nv_bfloat162*>(&t), hz);
    return *reinterpret_cast<const uint32_t*>(&out);
}
__device__ __forceinline__ float gelu_grad(float z, float t) {
    return fmaf(0.5f, 1.f + t, 0.5f * z * (1.f - t * t) * kGeluK * fmaf(3.f * kGeluA, z * z, 1.f));
}

__device__ __forceinline__ void st_row_chunk(uint8_t* tile, uint32_t row, uint32_t col, uint32_t sbo, const float* v) {
    *reinterpret_cast<uint4*>(tile + tc::tile_offset(row, col, sbo)) = tc::pack_bf16x8(v);
}

// Stage [W1 | b1] and [W2 | b2] as BF16 tiles and the FP32 vectors; write this thread's row of
// A1's constant columns (the ones column and the zero padding).
__device__ __forceinline__ void stage_weights(const float* __restrict__ net, uint8_t* w1s, uint8_t* w2s, float* w3,
                                              float* b3, float* mean, float* istd, uint8_t* a1s) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < kHid * 32; e += nt) {
        const int j = e >> 5, k = e & 31;
        const float v = k < kIn ? net[oW1 + j * kIn + k] : (k == kIn ? net[oB1 + j] : 0.f);
        *reinterpret_cast<__nv_bfloat16*>(w1s + tc::tile_offset(j, k, kSboW1)) = __float2bfloat16_rn(v);
    }
    for (int e = tid; e < kHid * 80; e += nt) {
        const int j = e / 80, i = e % 80;
        const float v = i < kHid ? net[oW2 + j * kHid + i] : (i == kHid ? net[oB2 + j] : 0.f);
        *reinterpret_cast<__nv_bfloat16*>(w2s + tc::tile_offset(j, i, kSboW2)) = __float2bfloat16_rn(v);
    }
    for (int e = tid; e < kHid; e += nt) w3[e] = net[oW3 + e];
    for (int e = tid; e < kIn; e += nt) {
        mean[e] = net[oMean + e];
        istd[e] = net[oInvStd + e];
    }
    if (tid == 0) *b3 = net[oB3];
    float v[8] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    st_row_chunk(a1s, tid, 64, kSboA1, v);
    v[0] = 0.f;
    st_row_chunk(a1s, tid, 72, kSboA1, v);
}

// One warp polls the MMA's mbarrier; the others wait at the block barrier, which issues nothing
// while it waits (polling from every warp takes issue slots from the other resident blocks).
__device__ __forceinline__ bool wait_mma(uint64_t* bar, uint32_t& phase, int* err) {
    bool ok = true;
    if (threadIdx.x < 32) ok = tc::mbar_wait(bar, phase, kWaitLimit);
    const bool failed = __syncthreads_or(!ok) != 0;
    if (!failed) phase ^= 1u;
    if (failed && threadIdx.x == 0) atomicExch(err, 1);
    tc::fence_after_sync();
    return !failed;
}

// Inference of one tile: X (this thread's row written by the caller) -> y of this thread's row.
// 64 TMEM columns (Z1, then Z2); returns false if a tensor-core wait gave up.
struct InferTile {
    uint8_t* a1s;
    uint32_t sX, sA1, sW1, sW2, tmem, lane_addr;
    uint64_t* bar;
    const float* w3;
    float b3;
};

__device__ __forceinline__ bool infer_tile(const InferTile& it, uint32_t& phase, int* err, float& y) {
    const int tid = threadIdx.x;
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
        tc::fence_after_sync();
        for (int s = 0; s < 2; ++s)
            tc::mma_bf16(it.tmem, tc::desc_kmajor(it.sX, kSboX, s), tc::desc_kmajor(it.sW1, kSboW1, s), kIdescFwd,
                         s > 0);
        tc::commit(it.bar);
    }
    if (!wait_mma(it.bar, phase, err)) return false;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float v[16];
        tc::tmem_ld16(it.tmem + it.lane_addr + 16 * c, v);
        uint4 lo, hi;
        lo.x = gelu_bf16x2(v[0], v[1]);
        lo.y = gelu_bf16x2(v[2], v[3]);
        lo.z = gelu_bf16x2(v[4], v[5]);
        lo.w = gelu_bf16x2(v[6], v[7]);
        hi.x = gelu_bf16x2(v[8], v[9]);
        hi.y = gelu_bf16x2(v[10], v[11]);
        hi.z = gelu_bf16x2(v[12], v[13]);
        hi.w = gelu_bf16x2(v[14], v[15]);
        *reinterpret_cast<uint4*>(it.a1s + tc::tile_offset(tid, 16 * c, kSboA1)) = lo;
        *reinterpret_cast<uint4*>(it.a1s + tc::tile_offset(tid, 16 * c + 8, kSboA1)) = hi;
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
        tc::fence_after_sync();
        for (int s = 0; s < 5; ++s)
            tc::mma_bf16(it.tmem, tc::desc_kmajor(it.sA1, kSboA1, s), tc::desc_kmajor(it.sW2, kSboW2, s), kIdescFwd,
                         s > 0);
        tc::commit(it.bar);
    }
    if (!wait_mma(it.bar, phase, err)) return false;
    float acc = it.b3;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float v[16];
        tc::tmem_ld16(it.tmem + it.lane_addr + 16 * c, v);
#pragma unroll
        for (int i = 0; i < 16; i += 4) {
            // w3 four at a time (one 128-bit shared load, the same address for every thread)
            const float4 w = *reinterpret_cast<const float4*>(it.w3 + 16 * c + i);
            const uint32_t g0 = gelu_bf16x2(v[i], v[i + 1]), g1 = gelu_bf16x2(v[i + 2], v[i + 3]);
            const float2 a0 = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&g0));
            const float2 a1 = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&g1));
            acc = fmaf(a0.x, w.x, acc);
            acc = fmaf(a0.y, w.y, acc);
            acc = fmaf(a1.x, w.z, acc);
            acc = fmaf(a1.y, w.w, acc);
        }
    }
    y = acc;
    return true;
}

// ---------------------------------------------------------------- features
// The 24 inputs of a D3Q19 node from its density and non-equilibrium populations (unscaled):
// the 19 MRT moments of f - feq over rho (the conserved four are zero), tr S, S:S, tr(Sd^3),
// |Sd| and the Cs = 0.1 Smagorinsky increment, S = -3 Pi / (2 rho tau0).
// spp (optional) receives sqrt(2 Pi:Pi), the stress norm of the relaxation formula.
// `unscale` multiplies neq first (the inverse storage scale for scaled deviations).
__device__ __forceinline__ void features(float rho, const float* neq, float tau0, float* x, float* spp = nullptr,
                                         float unscale = 1.f) {
    // moments M neq through sums / differences of opposite pairs (rows of lbm_d3q19.h:98-167)
    const float* n = neq;
    const float S1 = n[1] + n[2], D1 = n[1] - n[2];
    const float S2 = n[3] + n[4], D2 = n[3] - n[4];
    const float S3 = n[5] + n[6], D3 = n[5] - n[6];
    const float S4 = n[7] + n[10], D4 = n[7] - n[10];
    const float S5 = n[8] + n[9], D5 = n[8] - n[9];
    const float S6 = n[11] + n[14], D6 = n[11] - n[14];
    const float S7 = n[12] + n[13], D7 = n[12] - n[13];
    const float S8 = n[15] + n[18], D8 = n[15] - n[18];
    const float S9 = n[16] + n[17], D9 = n[16] - n[17];
    const float Sa = S1 + S2 + S3;
    const float Sxy = S4 + S5, Sxz = S6 + S7, Syz = S8 + S9;
    const float Sd = Sxy + Sxz + Syz;
    const float X1 = D4 - D5, X2 = D6 - D7, Y1 = D4 + D5, Y2 = D8 - D9, Z1 = D6 + D7, Z2 = D8 + D9;
    const float ir = unscale / rho;
    // mass and momentum of f - feq vanish (the collision conserves them): exact zero inputs,
    // not rounding noise that an input normalisation would amplify
    x[0] = 0.f;
    x[3] = 0.f;
    x[5] = 0.f;
    x[7] = 0.f;
    x[1] = (-30.f * n[0] - 11.f * Sa + 8.f * Sd) * ir;
    x[2] = (12.f * n[0] - 4.f * Sa + Sd) * ir;
    x[4] = (-4.f * D1 + X1 + X2) * ir;
    x[6] = (-4.f * D2 + Y1 + Y2) * ir;
    x[8] = (-4.f * D3 + Z1 + Z2) * ir;
    x[9] = (2.f * S1 - S2 - S3 + Sxy + Sxz - 2.f * Syz) * ir;
    x[10] = (-4.f * S1 + 2.f * (S2 + S3) + Sxy + Sxz - 2.f * Syz) * ir;
    x[11] = (S2 - S3 + Sxy - Sxz) * ir;
    x[12] = (-2.f * S2 + 2.f * S3 + Sxy - Sxz) * ir;
    x[13] = (S4 - S5) * ir;
    x[14] = (S8 - S9) * ir;
    x[15] = (S6 - S7) * ir;
    x[16] = (X1 - X2) * ir;
    x[17] = (-Y1 + Y2) * ir;
    x[18] = (Z1 - Z2) * ir;
    // non-equilibrium stress xx yy zz xy xz yz
    const float p[6] = {unscale * (S1 + S4 + S5 + S6 + S7), unscale * (S2 + S4 + S5 + S8 + S9),
                        unscale * (S3 + S6 + S7 + S8 + S9), unscale * (S4 - S5), unscale * (S6 - S7),
                        unscale * (S8 - S9)};
    const float k = -1.5f / (rho * tau0);
    float s[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) s[i] = k * p[i];
    const float tr = s[0] + s[1] + s[2];
    const float a = s[0] - tr / 3.f, b = s[1] - tr / 3.f, c = s[2] - tr / 3.f, d = s[3], e = s[4], g = s[5];
    const float ss = s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + 2.f * (d * d + e * e + g * g);
    const float det = a * (b * c - g * g) - d * (d * c - g * e) + e * (d * g - b * e);
    const float sd2 = a * a + b * b + c * c + 2.f * (d * d + e * e + g * g);
    const float pp = p[0] * p[0] + p[1] * p[1] + p[2] * p[2] + 2.f * (p[3] * p[3] + p[4] * p[4] + p[5] * p[5]);
    x[19] = tr;
    x[20] = ss;
    x[21] = 3.f * det;
    x[22] = sqrtf(2.f * sd2);
    const float s2 = sqrtf(2.f * pp);
    x[23] = 0.5f * (sqrtf(tau0 * tau0 + 18.f * kCUnit * s2) - tau0);
    if (spp) *spp = s2;
}

}  // namespace closure
}  // namespace zl
