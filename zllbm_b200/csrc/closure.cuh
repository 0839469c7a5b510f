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
// W1 [64 x 32], W2 [64 x 64]
constexpr uint32_t kSboX = 512, kSboA1 = 1280, kSboDz = 2048, kSboW1 = 512, kSboW2 = 1024;
constexpr uint32_t kBytesX = 128 * kSboX / 8, kBytesA1 = 128 * kSboA1 / 8, kBytesDz = 128 * kSboDz / 8,
                   kBytesW1 = 64 * kSboW1 / 8, kBytesW2 = 64 * kSboW2 / 8;
// every descriptor stays inside its buffer
static_assert(tc::extent_kmajor(128, kSboX, 2) <= kBytesX, "X as A (K = 32)");
static_assert(tc::extent_mnmajor(32, kSboX, 8) <= kBytesX, "X as B of dW1 (N = 32, K = 128)");
static_assert(tc::extent_kmajor(128, kSboA1, 4) <= kBytesA1, "A1 as A (K = 64)");
static_assert(tc::extent_mnmajor(80, kSboA1, 8) <= kBytesA1, "A1 as B of dW2 (N = 80, K = 128)");
static_assert(tc::extent_kmajor(128, kSboDz, 4) <= kBytesDz, "dZ2 as A of dA1 (K = 64)");
static_assert(tc::extent_mnmajor(128, kSboDz, 8) <= kBytesDz, "dZ as A of dW (M = 128, K = 128)");
static_assert(tc::extent_kmajor(64, kSboW1, 2) <= kBytesW1, "W1 as B (N = 64, K = 32)");
static_assert(tc::extent_kmajor(64, kSboW2, 4) <= kBytesW2, "W2 as B (N = 64, K = 64)");
static_assert(tc::extent_mnmajor(64, kSboW2, 4) <= kBytesW2, "W2^T as B of dA1 (N = 64, K = 64)");

// inference keeps A1 without the ones column: 64 columns, row groups 1024 B apart
constexpr uint32_t kSboA1f = 1024, kBytesA1f = 128 * kSboA1f / 8;
static_assert(tc::extent_kmajor(128, kSboA1f, 4) <= kBytesA1f, "A1 as A of the inference (K = 64)");

constexpr uint32_t kIdescFwd = tc::idesc_bf16(128, 64, false, false);   // X W1^T, A1 W2^T
constexpr uint32_t kIdescDa1 = tc::idesc_bf16(128, 64, false, true);    // dZ2 W2
constexpr uint32_t kIdescDw2 = tc::idesc_bf16(128, 80, true, true);     // dZ2^T [A1 | 1]
constexpr uint32_t kIdescDw1 = tc::idesc_bf16(128, 32, true, true);     // dZ1^T [X | 1]

__device__ __forceinline__ float gelu(float z, float& t) {
    t = tanhf(kGeluK * fmaf(kGeluA * z, z * z, z));
    return 0.5f * z * (1.f + t);
}
// inference: the tanh of the same formula by the hardware approximation (tanh.approx.f32)
__device__ __forceinline__ float gelu_fast(float z) {
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(kGeluK * fmaf(kGeluA * z, z * z, z)));
    return 0.5f * z * (1.f + t);
}
__device__ __forceinline__ float gelu_grad(float z, float t) {
    return fmaf(0.5f, 1.f + t, 0.5f * z * (1.f - t * t) * kGeluK * fmaf(3.f * kGeluA, z * z, 1.f));
}

__device__ __forceinline__ void st_row_chunk(uint8_t* tile, uint32_t row, uint32_t col, uint32_t sbo, const float* v) {
    *reinterpret_cast<uint4*>(tile + tc::tile_offset(row, col, sbo)) = tc::pack_bf16x8(v);
}

// Stage W1 and W2 as BF16 tiles (W1's columns 24 .. 31 zero) and the FP32 vectors.
__device__ __forceinline__ void stage_weights(const float* __restrict__ net, uint8_t* w1s, uint8_t* w2s, float* b1,
                                              float* b2, float* w3, float* b3, float* mean, float* istd) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < kHid * 32; e += nt) {
        const int j = e >> 5, k = e & 31;
        *reinterpret_cast<__nv_bfloat16*>(w1s + tc::tile_offset(j, k, kSboW1)) =
            __float2bfloat16_rn(k < kIn ? net[oW1 + j * kIn + k] : 0.f);
    }
    for (int e = tid; e < kHid * kHid; e += nt) {
        const int j = e >> 6, i = e & 63;
        *reinterpret_cast<__nv_bfloat16*>(w2s + tc::tile_offset(j, i, kSboW2)) = __float2bfloat16_rn(net[oW2 + e]);
    }
    for (int e = tid; e < kHid; e += nt) {
        b1[e] = net[oB1 + e];
        b2[e] = net[oB2 + e];
        w3[e] = net[oW3 + e];
    }
    for (int e = tid; e < kIn; e += nt) {
        mean[e] = net[oMean + e];
        istd[e] = net[oInvStd + e];
    }
    if (tid == 0) *b3 = net[oB3];
}

// ---------------------------------------------------------------- features
// The 24 inputs of a D3Q19 node from its density and non-equilibrium populations (unscaled):
// the 19 MRT moments of f - feq over rho (the conserved four are zero), tr S, S:S, tr(Sd^3),
// |Sd| and the Cs = 0.1 Smagorinsky increment, S = -3 Pi / (2 rho tau0).
// spp (optional) receives sqrt(2 Pi:Pi), the stress norm of the relaxation formula.
__device__ __forceinline__ void features(float rho, const float* neq, float tau0, float* x, float* spp = nullptr) {
    using Tb = Tables<D3Q19>;
    const float ir = 1.f / rho;
#pragma unroll
    for (int k = 0; k < 19; ++k) {
        // mass and momentum of f - feq vanish (the collision conserves them): exact zero inputs,
        // not rounding noise that an input normalisation would amplify
        if (k == 0 || k == 3 || k == 5 || k == 7) {
            x[k] = 0.f;
            continue;
        }
        float m = 0.f;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const int c = Tb::M(k, q);
            if (c == 1) m += neq[q];
            else if (c == -1) m -= neq[q];
            else if (c != 0) m = fmaf((float)c, neq[q], m);
        }
        x[k] = m * ir;
    }
    float p[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // xx yy zz xy xz yz
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        const int cx = Tb::cx(q), cy = Tb::cy(q), cz = Tb::cz(q);
        if (cx) p[0] += neq[q];
        if (cy) p[1] += neq[q];
        if (cz) p[2] += neq[q];
        if (cx * cy) p[3] += cx * cy > 0 ? neq[q] : -neq[q];
        if (cx * cz) p[4] += cx * cz > 0 ? neq[q] : -neq[q];
        if (cy * cz) p[5] += cy * cz > 0 ? neq[q] : -neq[q];
    }
    const float k = -1.5f * ir / tau0;
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
