// Learned LES closure on the device: the fused forward + backward tensor-core training kernel,
// the Adam update, the tensor-core forward pass, and the kernels that build training data from
// a fine level (box filter, subgrid-stress targets, features).  Full-box level I/O (set
// equilibrium, read macros from dense device arrays) lives here too.
//
// None of this has a counterpart in the reference; its relaxation formula is the reference's
// Smagorinsky increment (lbm_project/les_models/lbm_les_smagorinsky.cpp:22-94).
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "closure.cuh"
#include "closure_launch.cuh"
#include "zllbm_b200.h"

namespace zl {
namespace closure {

// ---------------------------------------------------------------- training
// Shared memory of the training kernel (bytes)
constexpr uint32_t kTrX = 0, kTrA1 = kTrX + kBytesX, kTrDz2 = kTrA1 + kBytesA1, kTrDz1 = kTrDz2 + kBytesDz,
                   kTrW1 = kTrDz1 + kBytesDz, kTrW2 = kTrW1 + kBytesW1, kTrF = kTrW2 + kBytesW2,
                   kTrBar = kTrF + 2048, kTrSmem = kTrBar + 64;
// TMEM columns: Z1 [0, 64), Z2 then dA1 [64, 128), dW2 | db2 [128, 208), dW1 | db1 [208, 240)
constexpr uint32_t kTmemCols = 256, kColZ1 = 0, kColZ2 = 64, kColDw2 = 128, kColDw1 = 208;

// One CTA of 128 threads per tile of 128 samples (thread = sample = TMEM lane).  Per tile:
//   MMA1  Z1 = X W1^T               MMA2  Z2 = A1 W2^T
//   MMA3  dA1 = dZ2 W2              MMA4  [dW2 | db2] += dZ2^T [A1 | 1]
//   MMA5  [dW1 | db1] += dZ1^T [X | 1]
// with the epilogues (bias, GELU, output, loss, dZ) on the CUDA cores between them.  The weight
// gradients accumulate in TMEM over the CTA's tiles and are added to `grad` once at the end.
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(128, 1) mlp_train_kernel(const float* __restrict__ net, const float* __restrict__ x,
                                                           const float* __restrict__ target, long long n, float inv_n,
                                                           float* __restrict__ grad, float* __restrict__ loss,
                                                           int* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float* fs = reinterpret_cast<float*>(sm + kTrF);
    float *w3 = fs + 128, *b3 = fs + 192, *mean = fs + 200, *istd = fs + 224;
    float* red = fs + 256;  // dw3 [64], db3, loss
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kTrBar);
    uint32_t* tbase = reinterpret_cast<uint32_t*>(sm + kTrBar + 8);

    stage_weights(net, sm + kTrW1, sm + kTrW2, w3, b3, mean, istd, sm + kTrA1);
    if (tid < 66) red[tid] = 0.f;
    {
        // the zero halves of the dZ tiles
        const float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (int c = 64; c < 128; c += 8) {
            st_row_chunk(sm + kTrDz2, tid, c, kSboDz, v);
            st_row_chunk(sm + kTrDz1, tid, c, kSboDz, v);
        }
    }
    if (warp == 0) tc::tmem_alloc(tbase, kTmemCols);
    if (tid == 0) tc::mbar_init(bar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tbase;
    const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
    const uint32_t sX = tc::smem_u32(sm + kTrX), sA1 = tc::smem_u32(sm + kTrA1), sDz2 = tc::smem_u32(sm + kTrDz2),
                   sDz1 = tc::smem_u32(sm + kTrDz1), sW1 = tc::smem_u32(sm + kTrW1), sW2 = tc::smem_u32(sm + kTrW2);
    uint32_t phase = 0;
    float loss_acc = 0.f, db3_acc = 0.f;
    bool first = true, ok = true;
    const long long tiles = (n + kTile - 1) / kTile;

    for (long long tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const long long g = tile * kTile + tid;
        const bool valid = g < n;
        {
            float v[32];
#pragma unroll
            for (int k = 0; k < kIn; ++k) v[k] = valid ? (x[g * kIn + k] - mean[k]) * istd[k] : 0.f;
            v[24] = 1.f;
#pragma unroll
            for (int k = 25; k < 32; ++k) v[k] = 0.f;
#pragma unroll
            for (int c = 0; c < 4; ++c) st_row_chunk(sm + kTrX, tid, 8 * c, kSboX, v + 8 * c);
        }
        const float t = valid ? target[g] : 0.f;

        // MMA1: Z1 = [X | 1] [W1 | b1]^T
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            for (int s = 0; s < 2; ++s)
                tc::mma_bf16(tmem + kColZ1, tc::desc_kmajor(sX, kSboX, s), tc::desc_kmajor(sW1, kSboW1, s), kIdescFwd,
                             s > 0);
            tc::commit(bar);
        }
        if (!(ok = wait_mma(bar, phase, err))) break;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float v[16];
            tc::tmem_ld16(tmem + lane_addr + kColZ1 + 16 * c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float th;
                v[i] = gelu(v[i], th);
            }
            st_row_chunk(sm + kTrA1, tid, 16 * c, kSboA1, v);
            st_row_chunk(sm + kTrA1, tid, 16 * c + 8, kSboA1, v + 8);
        }

        // MMA2: Z2 = [A1 | 1] [W2 | b2]^T
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            for (int s = 0; s < 5; ++s)
                tc::mma_bf16(tmem + kColZ2, tc::desc_kmajor(sA1, kSboA1, s), tc::desc_kmajor(sW2, kSboW2, s),
                             kIdescFwd, s > 0);
            tc::commit(bar);
        }
        if (!(ok = wait_mma(bar, phase, err))) break;
        float y = *b3;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float v[16];
            tc::tmem_ld16(tmem + lane_addr + kColZ2 + 16 * c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float th;
                y = fmaf(gelu(v[i], th), w3[16 * c + i], y);
            }
        }
        const float e = valid ? y - t : 0.f;
        loss_acc = fmaf(e, e, loss_acc);
        const float dy = 2.f * e * inv_n;
        db3_acc += dy;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float v[16];
            tc::tmem_ld16(tmem + lane_addr + kColZ2 + 16 * c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int j = 16 * c + i;
                const float z = v[i];
                float th;
                const float a2 = gelu(z, th);
                const float s = warp_sum(dy * a2);
                if (lane == 0) atomicAdd(red + j, s);
                v[i] = dy * w3[j] * gelu_grad(z, th);
            }
            st_row_chunk(sm + kTrDz2, tid, 16 * c, kSboDz, v);
            st_row_chunk(sm + kTrDz2, tid, 16 * c + 8, kSboDz, v + 8);
        }

        // MMA3: dA1 = dZ2 W2 (into the Z2 columns), MMA4: [dW2 | db2] += dZ2^T [A1 | 1]
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            for (int s = 0; s < 4; ++s)
                tc::mma_bf16(tmem + kColZ2, tc::desc_kmajor(sDz2, kSboDz, s), tc::desc_mnmajor(sW2, kSboW2, s),
                             kIdescDa1, s > 0);
            for (int s = 0; s < 8; ++s)
                tc::mma_bf16(tmem + kColDw2, tc::desc_mnmajor(sDz2, kSboDz, s), tc::desc_mnmajor(sA1, kSboA1, s),
                             kIdescDw2, !first || s > 0);
            tc::commit(bar);
        }
        if (!(ok = wait_mma(bar, phase, err))) break;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float da[16], z1[16];
            tc::tmem_ld16(tmem + lane_addr + kColZ2 + 16 * c, da);
            tc::tmem_ld16(tmem + lane_addr + kColZ1 + 16 * c, z1);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const float z = z1[i];
                float th;
                gelu(z, th);
                da[i] *= gelu_grad(z, th);
            }
            st_row_chunk(sm + kTrDz1, tid, 16 * c, kSboDz, da);
            st_row_chunk(sm + kTrDz1, tid, 16 * c + 8, kSboDz, da + 8);
        }

        // MMA5: [dW1 | db1] += dZ1^T [X | 1]
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            for (int s = 0; s < 8; ++s)
                tc::mma_bf16(tmem + kColDw1, tc::desc_mnmajor(sDz1, kSboDz, s), tc::desc_mnmajor(sX, kSboX, s),
                             kIdescDw1, !first || s > 0);
            tc::commit(bar);
        }
        if (!(ok = wait_mma(bar, phase, err))) break;
        first = false;
    }
    if (!ok) {
        // a wait gave up: give the tensor cores one more bounded wait before TMEM is released
        tc::mbar_wait(bar, phase, kWaitLimit);
    }

    // weight gradients: rows j = 0 .. 63 of the accumulators sit in TMEM lanes 0 .. 63
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (ok && !first && warp < 2) {
        const int j = tid;
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            float v[16];
            tc::tmem_ld16(tmem + lane_addr + kColDw2 + 16 * c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int col = 16 * c + i;
                if (col < kHid) atomicAdd(grad + oW2 + j * kHid + col, v[i]);
                else if (col == kHid) atomicAdd(grad + oB2 + j, v[i]);
            }
        }
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            float v[16];
            tc::tmem_ld16(tmem + lane_addr + kColDw1 + 16 * c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int col = 16 * c + i;
                if (col < kIn) atomicAdd(grad + oW1 + j * kIn + col, v[i]);
                else if (col == kIn) atomicAdd(grad + oB1 + j, v[i]);
            }
        }
    }
    loss_acc = warp_sum(loss_acc);
    db3_acc = warp_sum(db3_acc);
    if (lane == 0) {
        atomicAdd(red + 64, db3_acc);
        atomicAdd(red + 65, loss_acc);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (ok && tid < kHid) atomicAdd(grad + oW3 + tid, red[tid]);
    if (ok && tid == 0) {
        atomicAdd(grad + oB3, red[64]);
        atomicAdd(loss, red[65]);
    }
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kTmemCols);
    }
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
}

// ---------------------------------------------------------------- forward (inference)
// Shared memory of the inference kernels (bytes); TMEM: 64 columns, Z1 then Z2
constexpr uint32_t kFwX = 0, kFwA1 = kFwX + kBytesX, kFwW1 = kFwA1 + kBytesA1, kFwW2 = kFwW1 + kBytesW1,
                   kFwF = kFwW2 + kBytesW2, kFwBar = kFwF + 1024, kFwSmem = kFwBar + 64;
constexpr uint32_t kFwSmemLaunch = kFwSmem;
constexpr uint32_t kInferCols = 64;
constexpr int kMaxCtaPerSm = 512 / kInferCols;

// Set-up shared by the inference kernels: weights staged, TMEM allocated, barrier initialised.
__device__ __forceinline__ InferTile infer_setup(uint8_t* sm, const float* net, float*& mean, float*& istd) {
    const int warp = threadIdx.x >> 5;
    float* fs = reinterpret_cast<float*>(sm + kFwF);
    float *w3 = fs + 128, *b3 = fs + 192;
    mean = fs + 200;
    istd = fs + 224;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kFwBar);
    uint32_t* tbase = reinterpret_cast<uint32_t*>(sm + kFwBar + 8);
    stage_weights(net, sm + kFwW1, sm + kFwW2, w3, b3, mean, istd, sm + kFwA1);
    if (warp == 0) tc::tmem_alloc(tbase, kInferCols);
    if (threadIdx.x == 0) tc::mbar_init(bar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    InferTile it;
    it.a1s = sm + kFwA1;
    it.sX = tc::smem_u32(sm + kFwX);
    it.sA1 = tc::smem_u32(sm + kFwA1);
    it.sW1 = tc::smem_u32(sm + kFwW1);
    it.sW2 = tc::smem_u32(sm + kFwW2);
    it.tmem = *tbase;
    it.lane_addr = (uint32_t)(warp * 32) << 16;
    it.bar = bar;
    it.w3 = w3;
    it.b3 = *b3;
    return it;
}

__device__ __forceinline__ void infer_teardown(const InferTile& it, bool ok, uint32_t phase) {
    if (!ok) tc::mbar_wait(it.bar, phase, kWaitLimit);  // give the tensor cores a last bounded wait
    tc::fence_before_sync();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(it.tmem, kInferCols);
    }
}

// Write this thread's normalised feature row [x_hat | 1 | 0] into the X tile.
__device__ __forceinline__ void write_x_row(uint8_t* xs, const float* x, const float* mean, const float* istd,
                                            bool valid) {
    float v[32];
#pragma unroll
    for (int k = 0; k < kIn; ++k) v[k] = valid ? (x[k] - mean[k]) * istd[k] : 0.f;
    v[kIn] = 1.f;
#pragma unroll
    for (int k = kIn + 1; k < 32; ++k) v[k] = 0.f;
#pragma unroll
    for (int c = 0; c < 4; ++c) st_row_chunk(xs, threadIdx.x, 8 * c, kSboX, v + 8 * c);
}

__global__ void __launch_bounds__(128) mlp_forward_kernel(const float* __restrict__ net, const float* __restrict__ x,
                                                          long long n, float* __restrict__ out, int* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t sm[];
    float *mean, *istd;
    const InferTile it = infer_setup(sm, net, mean, istd);
    uint32_t phase = 0;
    bool ok = true;
    const long long tiles = (n + kTile - 1) / kTile;
    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const long long g = tile * kTile + threadIdx.x;
        const bool valid = g < n;
        float xv[kIn];
#pragma unroll
        for (int k = 0; k < kIn; ++k) xv[k] = valid ? x[g * kIn + k] : 0.f;
        write_x_row(sm + kFwX, xv, mean, istd, valid);
        float y;
        if (!(ok = infer_tile(it, phase, err, y))) break;
        if (valid) out[g] = y;
    }
    infer_teardown(it, ok, phase);
}

// ---------------------------------------------------------------- full-box I/O, features, filter
__device__ __forceinline__ Coord box_coord(const LevelGeom& geo, long long i) {
    Coord c;
    c.x[0] = (int)(i % geo.n[0]);
    const long long r = i / geo.n[0];
    c.x[1] = (int)(r % geo.n[1]);
    c.x[2] = (int)(r / geo.n[1]);
    return c;
}

template <class S>
__global__ void set_equilibrium_kernel(S* __restrict__ f, LevelGeom geo, StepParams p, int even,
                                       const float* __restrict__ rho, const float* __restrict__ u, long long nn) {
    using Tb = Tables<D3Q19>;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const Coord c = box_coord(geo, i);
    const float r = rho[i], ux = u[i * 3], uy = u[i * 3 + 1], uz = u[i * 3 + 2];
    const float usq15 = 1.5f * (ux * ux + uy * uy + uz * uz);
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const float cu = signed_dot<D3Q19>(q, ux, uy, uz);
        const float w = (float)Tb::w(q);
        // feq - w = w (rho - 1) + w rho (3 cu + 4.5 cu^2 - 1.5 u^2)
        const float d = w * fmaf(r, fmaf(cu, fmaf(4.5f, cu, 3.f), -usq15), r - 1.f);
        Storage<S>::store(f + post_stream_slot<D3Q19>(geo, c, q, even), d, p);
    }
}

template <class S>
__device__ __forceinline__ void load_node(const S* f, const LevelGeom& geo, const Coord& c, int even, float* d) {
#pragma unroll
    for (int q = 0; q < 19; ++q) d[q] = Storage<S>::load_raw(f + post_stream_slot<D3Q19>(geo, c, q, even));
}

template <class S>
__global__ void get_macros_kernel(const S* __restrict__ f, LevelGeom geo, StepParams p, int even,
                                  float* __restrict__ rho, float* __restrict__ u, long long nn) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= nn) return;
    float d[19], neq[19], mac[4];
    load_node(f, geo, box_coord(geo, i), even, d);
    feq_neq_dev<D3Q19>(d, neq, p.scale, p.inv_scale, mac);
    rho[i] = mac[0];
    u[i * 3] = mac[1];
    u[i * 3 + 1] = mac[2];
    u[i * 3 + 2] = mac[3];
}

// FP64 storage (absolute populations): feq in the reference's arithmetic order from the FP32
// fields, and rho / u by the reference's macro rule, rounded to FP32 on output.
__global__ void set_equilibrium_f64_kernel(double* __restrict__ f, LevelGeom geo, int even,
                                           const float* __restrict__ rho, const float* __restrict__ u, long long nn) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const Coord c = box_coord(geo, i);
    double feq[19];
    feq_exact<D3Q19>((double)rho[i], (double)u[i * 3], (double)u[i * 3 + 1], (double)u[i * 3 + 2], feq);
#pragma unroll
    for (int q = 0; q < 19; ++q) f[post_stream_slot<D3Q19>(geo, c, q, even)] = feq[q];
}

__global__ void get_macros_f64_kernel(const double* __restrict__ f, LevelGeom geo, int even,
                                      float* __restrict__ rho, float* __restrict__ u, long long nn) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const Coord c = box_coord(geo, i);
    double v[19], r, ux, uy, uz;
#pragma unroll
    for (int q = 0; q < 19; ++q) v[q] = f[post_stream_slot<D3Q19>(geo, c, q, even)];
    macro_exact<D3Q19>(v, r, ux, uy, uz);
    rho[i] = (float)r;
    u[i * 3] = (float)ux;
    u[i * 3 + 1] = (float)uy;
    u[i * 3 + 2] = (float)uz;
}

template <class S>
__global__ void features_kernel(const S* __restrict__ f, LevelGeom geo, StepParams p, int even,
                                float* __restrict__ x, long long nn) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= nn) return;
    float d[19], neq[19], mac[4], v[kIn];
    load_node(f, geo, box_coord(geo, i), even, d);
    feq_neq_dev<D3Q19>(d, neq, p.scale, p.inv_scale, mac);
    features(mac[0], neq, (float)p.tau, v, nullptr, p.inv_scale);
#pragma unroll
    for (int k = 0; k < kIn; ++k) x[i * kIn + k] = v[k];
}

// One thread per factor^3 block of nodes: block means of rho, u, u_a u_b and f - feq.
template <class S>
__global__ void filter_kernel(const S* __restrict__ f, LevelGeom geo, StepParams p, int even, int factor, int ncx,
                              int ncy, int ncz, float* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nc = (long long)ncx * ncy * ncz;
    if (i >= nc) return;
    const int X = (int)(i % ncx), Y = (int)((i / ncx) % ncy), Z = (int)(i / ((long long)ncx * ncy));
    float acc[29];
#pragma unroll
    for (int k = 0; k < 29; ++k) acc[k] = 0.f;
    for (int dz = 0; dz < factor; ++dz)
        for (int dy = 0; dy < factor; ++dy)
            for (int dx = 0; dx < factor; ++dx) {
                Coord c;
                c.x[0] = X * factor + dx;
                c.x[1] = Y * factor + dy;
                c.x[2] = Z * factor + dz;
                float d[19], neq[19], mac[4];
                load_node(f, geo, c, even, d);
                feq_neq_dev<D3Q19>(d, neq, p.scale, p.inv_scale, mac);
                acc[0] += mac[0];
                acc[1] += mac[1];
                acc[2] += mac[2];
                acc[3] += mac[3];
                acc[4] += mac[1] * mac[1];
                acc[5] += mac[2] * mac[2];
                acc[6] += mac[3] * mac[3];
                acc[7] += mac[1] * mac[2];
                acc[8] += mac[1] * mac[3];
                acc[9] += mac[2] * mac[3];
#pragma unroll
                for (int q = 0; q < 19; ++q) acc[10 + q] += neq[q] * p.inv_scale;
            }
    const float inv = 1.f / (float)(factor * factor * factor);
#pragma unroll
    for (int k = 0; k < 29; ++k) out[i * 29 + k] = acc[k] * inv;
}

// ---------------------------------------------------------------- training pairs
__device__ __forceinline__ long long wrap_index(int x, int y, int z, const int* n) {
    x = (x + n[0]) % n[0];
    y = (y + n[1]) % n[1];
    z = (z + n[2]) % n[2];
    return (long long)x + (long long)n[0] * (y + (long long)n[1] * z);
}

struct Grid3 {
    int n[3];
};

// Strain of the filtered field as the coarse lattice sees it, S = -3 factor Pi<f - feq> / (2 rho tau_f)
// (the fine non-equilibrium stress is -2/3 rho tau_f S_fine and S_coarse = factor S_fine), the exact
// subgrid stress, and the least-squares pieces of c over a node: num = tau^d : M, den = M : M,
// M = 2 |S| S.  Using the strain the collision itself estimates keeps the target consistent with
// the way the closure is applied.
__device__ __forceinline__ void filtered_strain(const float* cf, float tau_fine, int factor, float* s) {
    using Tb = Tables<D3Q19>;
    float p[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        const float n = cf[10 + q];
        const int cx = Tb::cx(q), cy = Tb::cy(q), cz = Tb::cz(q);
        if (cx) p[0] += n;
        if (cy) p[1] += n;
        if (cz) p[2] += n;
        if (cx * cy) p[3] += cx * cy > 0 ? n : -n;
        if (cx * cz) p[4] += cx * cz > 0 ? n : -n;
        if (cy * cz) p[5] += cy * cz > 0 ? n : -n;
    }
    const float k = -1.5f * (float)factor / (cf[0] * tau_fine);
#pragma unroll
    for (int i = 0; i < 6; ++i) s[i] = k * p[i];
}

__global__ void pairs_stage1_kernel(Grid3 g, const float* __restrict__ filt, float tau_fine, int factor,
                                    float* __restrict__ scratch) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nn = (long long)g.n[0] * g.n[1] * g.n[2];
    if (i >= nn) return;
    const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
    const float* c = filt + i * 29;
    float s[6], td[6];
    filtered_strain(c, tau_fine, factor, s);
    for (int k = 0; k < 6; ++k) td[k] = c[4 + k] - c[1 + pa[k]] * c[1 + pb[k]];
    const float tr = (td[0] + td[1] + td[2]) / 3.f;
    td[0] -= tr;
    td[1] -= tr;
    td[2] -= tr;
    const float ss = s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + 2.f * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
    const float smag = sqrtf(2.f * ss);
    float num = 0.f, den = 0.f;
    for (int k = 0; k < 6; ++k) {
        const float m = 2.f * smag * s[k];
        const float w = k < 3 ? 1.f : 2.f;
        num += w * td[k] * m;
        den += w * m * m;
    }
    scratch[i * 3] = num;
    scratch[i * 3 + 1] = den;
    scratch[i * 3 + 2] = smag;
}

__global__ void pairs_stage2_kernel(Grid3 g, const float* __restrict__ filt, const float* __restrict__ scratch,
                                    float tau_fine, float tau_coarse, int factor, float* __restrict__ xo,
                                    float* __restrict__ yo) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nn = (long long)g.n[0] * g.n[1] * g.n[2];
    if (i >= nn) return;
    const int x = (int)(i % g.n[0]), y = (int)((i / g.n[0]) % g.n[1]), z = (int)(i / ((long long)g.n[0] * g.n[1]));
    float num = 0.f, den = 0.f;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const long long j = wrap_index(x + dx, y + dy, z + dz, g.n);
                num += scratch[j * 3];
                den += scratch[j * 3 + 1];
            }
    num /= 27.f;
    den /= 27.f;
    const float c = den > 1e-30f ? -num / den : 0.f;  // no resolved strain: no constant to fit
    const float yv = fminf(fmaxf(c / kCUnit, 0.f), kYMax);
    const float tau_eff = tau_coarse + 3.f * kCUnit * yv * scratch[i * 3 + 2];
    const float r = (float)factor * tau_eff / tau_fine;
    const float* cf = filt + i * 29;
    float neq[19], v[kIn];
#pragma unroll
    for (int q = 0; q < 19; ++q) neq[q] = r * cf[10 + q];
    features(cf[0], neq, tau_coarse, v);
#pragma unroll
    for (int k = 0; k < kIn; ++k) xo[i * kIn + k] = v[k];
    yo[i] = yv;
}

// ---------------------------------------------------------------- fused collide-stream with the network
// The AA step of a full periodic box with the learned closure evaluated inside the collision:
// one persistent CTA of 128 threads per tile of 128 consecutive nodes; each thread loads its
// node's populations, writes its features into the X tile, the CTA runs the two tensor-core
// layers, and each thread relaxes with tau = tau0 + 0.5 (sqrt(tau0^2 + 18 c sqrt(2 Pi:Pi)) - tau0)
// and streams; c is also stored per node (c_node) for the steps that reuse it.  The grid is the
// number of CTAs that fit on the GPU (shared memory 37 KiB, TMEM 64 columns per CTA).
constexpr uint32_t kLsSmemLaunch = kFwSmem;

template <class S, int Coll, bool Odd>
__global__ void __launch_bounds__(128, 5) learned_step_kernel(S* __restrict__ f, LevelGeom geo, StepParams p,
                                                           const float* __restrict__ net, float fallback_c,
                                                           float* __restrict__ c_node, int* __restrict__ err,
                                                           FastDiv nx, FastDiv ny) {
    using Tb = Tables<D3Q19>;
    using St = Storage<S>;
    extern __shared__ __align__(1024) uint8_t sm[];
    float *mean, *istd;
    const InferTile it = infer_setup(sm, net, mean, istd);
    const int tid = threadIdx.x;
    const float tau0 = (float)p.tau;
    const long long nn = (long long)geo.n[0] * geo.n[1] * geo.n[2];
    const long long tiles = (nn + kTile - 1) / kTile;
    const long long st = geo.stride;
    uint32_t phase = 0;
    bool ok = true;

    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const long long i = tile * kTile + tid;
        const bool valid = i < nn;
        Coord c;
        {
            // node index -> coordinates (x fastest) by multiply-shift division (the box holds
            // fewer than 2^31 cells)
            const uint32_t ii = valid ? (uint32_t)i : 0u;
            const uint32_t r = nx.div(ii), zq = ny.div(r);
            c.x[0] = (int)(ii - r * (uint32_t)geo.n[0]);
            c.x[1] = (int)(r - zq * (uint32_t)geo.n[1]);
            c.x[2] = (int)zq;
        }
        // periodic neighbours of the node (the level wraps on every axis)
        int bx[3], row[3][3];
        {
            int by[3], bz[3];
#pragma unroll
            for (int d = -1; d <= 1; ++d) {
                bx[d + 1] = wrap_or_ghost(c.x[0] + d, geo.n[0], 0, 1);
                by[d + 1] = wrap_or_ghost(c.x[1] + d, geo.n[1], 0, 1);
                bz[d + 1] = wrap_or_ghost(c.x[2] + d, geo.n[2], 0, 1);
            }
#pragma unroll
            for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                for (int dz = 0; dz < 3; ++dz) row[dy][dz] = geo.a[0] * (by[dy] + geo.a[1] * bz[dz]);
        }
        auto cell = [&](int dx, int dy, int dz) -> int { return bx[dx + 1] + row[dy + 1][dz + 1]; };
        const int self = cell(0, 0, 0);
        float pre[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            if (!valid) pre[q] = 0.f;
            else if (Odd && q != 0) pre[q] = St::load_raw(f + Tb::opp(q) * st + cell(-Tb::cx(q), -Tb::cy(q), -Tb::cz(q)));
            else pre[q] = St::load_raw(f + q * st + self);
        }
        float pp;  // sqrt(2 Pi:Pi) of the unscaled non-equilibrium part
        float neq[19], mac[4];
        feq_neq_dev<D3Q19>(pre, neq, p.scale, p.inv_scale, mac);
        {
            float x[kIn];
            features(mac[0], neq, tau0, x, &pp, p.inv_scale);
            write_x_row(sm + kFwX, x, mean, istd, valid);
        }
        float y;
        if (!(ok = infer_tile(it, phase, err, y))) break;
        if (!valid) continue;
        const float cc = isfinite(y) ? kCUnit * fminf(fmaxf(y, 0.f), kYMax) : fallback_c;
        if (c_node) c_node[self] = cc;
        const float tau = tau0 + 0.5f * (sqrtf(fmaf(tau0, tau0, 18.f * cc * pp)) - tau0);
        const float omega = 1.f / tau;
        float post[19];
        if (Coll == kSrt) {
#pragma unroll
            for (int q = 0; q < 19; ++q) post[q] = fmaf(-omega, neq[q], pre[q]);
        } else {
            float lam[19];
#pragma unroll
            for (int k = 0; k < 19; ++k)
                lam[k] = Tb::s(k) > 0. ? ((float)Tb::s(k) - omega) / (float)row_norm2<D3Q19>(k) : 0.f;
            mrt_d3q19_dev(pre, neq, post, omega, lam);
        }
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            if (Odd && q != 0) St::store_raw(f + q * st + cell(Tb::cx(q), Tb::cy(q), Tb::cz(q)), post[q]);
            else St::store_raw(f + Tb::opp(q) * st + self, post[q]);
        }
    }
    infer_teardown(it, ok, phase);
}

template <class S>
static cudaError_t learned_step_s(int coll, bool odd, void* f, const LevelGeom& geo, const StepParams& p,
                                  const float* net, float fallback_c, float* c_node, int* err, cudaStream_t s) {
    static int grid[4] = {0, 0, 0, 0};
    auto launch = [&](auto kernel, int slot) -> cudaError_t {
        if (!grid[slot]) {
            cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLsSmemLaunch);
            if (e != cudaSuccess) return e;
            int dev = 0, sms = 0, regs_sm = 0, smem_sm = 0, reserved = 0;
            cudaFuncAttributes fa;
            if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
                (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
                (e = cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev)) != cudaSuccess ||
                (e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess ||
                (e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev)) != cudaSuccess ||
                (e = cudaFuncGetAttributes(&fa, kernel)) != cudaSuccess)
                return e;
            // resident CTAs per SM from registers (allocated per warp in units of 256), shared
            // memory, and TMEM (at most 512 / 64 so that no CTA waits for columns)
            const int regs_cta = 4 * ((fa.numRegs * 32 + 255) / 256 * 256);
            const int by_regs = regs_cta > 0 ? regs_sm / regs_cta : kMaxCtaPerSm;
            const int by_smem = smem_sm / (int)(kLsSmemLaunch + fa.sharedSizeBytes + reserved);
            int per_sm = by_regs < by_smem ? by_regs : by_smem;
            per_sm = per_sm < kMaxCtaPerSm ? per_sm : kMaxCtaPerSm;
            grid[slot] = sms * (per_sm > 0 ? per_sm : 1);
        }
        kernel<<<grid[slot], 128, kLsSmemLaunch, s>>>(static_cast<S*>(f), geo, p, net, fallback_c, c_node, err,
                                                      FastDiv::make((uint32_t)geo.n[0]),
                                                      FastDiv::make((uint32_t)geo.n[1]));
        return cudaGetLastError();
    };
    if (coll == kMrt)
        return odd ? launch(learned_step_kernel<S, kMrt, true>, 0) : launch(learned_step_kernel<S, kMrt, false>, 1);
    return odd ? launch(learned_step_kernel<S, kSrt, true>, 2) : launch(learned_step_kernel<S, kSrt, false>, 3);
}

// ---------------------------------------------------------------- launchers used by the API
template <class S>
static cudaError_t dispatch_box(int op, void* f, const LevelGeom& geo, const StepParams& p, int even, const float* a,
                                float* b, float* c, int factor, const int* nc, cudaStream_t s) {
    const long long nn = (long long)geo.n[0] * geo.n[1] * geo.n[2];
    const unsigned blocks = (unsigned)((nn + 255) / 256);
    switch (op) {
        case kBoxSetEq:
            set_equilibrium_kernel<S><<<blocks, 256, 0, s>>>((S*)f, geo, p, even, a, b, nn);
            break;
        case kBoxGetMacros:
            get_macros_kernel<S><<<blocks, 256, 0, s>>>((const S*)f, geo, p, even, b, c, nn);
            break;
        case kBoxFeatures:
            features_kernel<S><<<blocks, 256, 0, s>>>((const S*)f, geo, p, even, b, nn);
            break;
        case kBoxFilter: {
            const long long ncn = (long long)nc[0] * nc[1] * nc[2];
            filter_kernel<S><<<(unsigned)((ncn + 127) / 128), 128, 0, s>>>((const S*)f, geo, p, even, factor, nc[0],
                                                                            nc[1], nc[2], b);
            break;
        }
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace closure

cudaError_t closure_learned_step(int storage, int coll, bool odd, void* f, const LevelGeom& geo, const StepParams& p,
                                 const float* net, float fallback_c, float* c_node, int* err, cudaStream_t s) {
    using namespace closure;
    switch (storage) {
        case ZL_STORAGE_F32: return learned_step_s<float>(coll, odd, f, geo, p, net, fallback_c, c_node, err, s);
        case ZL_STORAGE_F16: return learned_step_s<__half>(coll, odd, f, geo, p, net, fallback_c, c_node, err, s);
        case ZL_STORAGE_BF16:
            return learned_step_s<__nv_bfloat16>(coll, odd, f, geo, p, net, fallback_c, c_node, err, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t closure_box_op(int op, int storage, void* f, const LevelGeom& geo, const StepParams& p, int even,
                           const float* a, float* b, float* c, int factor, const int* nc, cudaStream_t s) {
    using namespace closure;
    switch (storage) {
        case ZL_STORAGE_F32: return dispatch_box<float>(op, f, geo, p, even, a, b, c, factor, nc, s);
        case ZL_STORAGE_F16: return dispatch_box<__half>(op, f, geo, p, even, a, b, c, factor, nc, s);
        case ZL_STORAGE_BF16: return dispatch_box<__nv_bfloat16>(op, f, geo, p, even, a, b, c, factor, nc, s);
        case ZL_STORAGE_F64: {
            const long long nn = (long long)geo.n[0] * geo.n[1] * geo.n[2];
            const unsigned blocks = (unsigned)((nn + 255) / 256);
            if (op == kBoxSetEq)
                set_equilibrium_f64_kernel<<<blocks, 256, 0, s>>>((double*)f, geo, even, a, b, nn);
            else if (op == kBoxGetMacros)
                get_macros_f64_kernel<<<blocks, 256, 0, s>>>((const double*)f, geo, even, b, c, nn);
            else
                return cudaErrorInvalidValue;
            return cudaGetLastError();
        }
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace zl

// ---------------------------------------------------------------- C ABI (context-free part)
using namespace zl;
using namespace zl::closure;

struct zl_trainer {
    int device = 0;
    cudaStream_t stream = nullptr;      // stream the trainer issues on
    cudaStream_t own_stream = nullptr;  // the trainer's own stream
    float* w = nullptr;     // kFlat: weights (trainable part first) + normalisation
    float* g = nullptr;     // kTrainable gradients of the last step
    float* m = nullptr;     // Adam moments
    float* v = nullptr;
    float* loss = nullptr;  // sum of squared errors of the last step
    int* err = nullptr;
    long long t = 0;        // Adam step count
    long long last_n = 0;
};

static_assert(sizeof(zl_mlp) == sizeof(float) * kFlat, "zl_mlp layout");

static int train_attr_once(int device) {
    static std::mutex mu;
    static bool done[64] = {false};
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0 || device >= 64) return ZL_EINVAL;
    if (!done[device]) {
        if (cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrSmem) !=
                cudaSuccess ||
            cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kFwSmemLaunch) != cudaSuccess)
            return ZL_EDEVICE;
        done[device] = true;
    }
    return ZL_OK;
}

extern "C" {

int zl_trainer_create(const zl_mlp* init, int device, zl_trainer** out) {
    if (!init || !out) return ZL_EINVAL;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return ZL_EDEVICE;
    int rc = train_attr_once(device);
    if (rc) return rc;
    zl_trainer* tr = new zl_trainer();
    tr->device = device;
    bool ok = cudaStreamCreateWithFlags(&tr->own_stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(&tr->w, sizeof(float) * kFlat) == cudaSuccess &&
              cudaMalloc(&tr->g, sizeof(float) * kTrainable) == cudaSuccess &&
              cudaMalloc(&tr->m, sizeof(float) * kTrainable) == cudaSuccess &&
              cudaMalloc(&tr->v, sizeof(float) * kTrainable) == cudaSuccess &&
              cudaMalloc(&tr->loss, sizeof(float)) == cudaSuccess && cudaMalloc(&tr->err, sizeof(int)) == cudaSuccess;
    ok = ok && cudaMemcpy(tr->w, init, sizeof(float) * kFlat, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(tr->g, 0, sizeof(float) * kTrainable) == cudaSuccess &&
         cudaMemset(tr->m, 0, sizeof(float) * kTrainable) == cudaSuccess &&
         cudaMemset(tr->v, 0, sizeof(float) * kTrainable) == cudaSuccess &&
         cudaMemset(tr->loss, 0, sizeof(float)) == cudaSuccess && cudaMemset(tr->err, 0, sizeof(int)) == cudaSuccess;
    tr->stream = tr->own_stream;
    if (!ok) {
        zl_trainer_destroy(tr);
        return ZL_EDEVICE;
    }
    *out = tr;
    return ZL_OK;
}

int zl_trainer_set_stream(zl_trainer* tr, void* stream) {
    if (!tr) return ZL_EINVAL;
    if (cudaSetDevice(tr->device) != cudaSuccess || cudaStreamSynchronize(tr->stream) != cudaSuccess)
        return ZL_EDEVICE;
    tr->stream = stream ? static_cast<cudaStream_t>(stream) : tr->own_stream;
    return ZL_OK;
}

int zl_trainer_step(zl_trainer* tr, const float* x_device, const float* y_device, int64_t n, float lr) {
    if (!tr || !x_device || !y_device || n <= 0) return ZL_EINVAL;
    if (cudaSetDevice(tr->device) != cudaSuccess) return ZL_EDEVICE;
    cudaStream_t s = tr->stream;
    if (cudaMemsetAsync(tr->g, 0, sizeof(float) * kTrainable, s) != cudaSuccess ||
        cudaMemsetAsync(tr->loss, 0, sizeof(float), s) != cudaSuccess)
        return ZL_EDEVICE;
    const long long tiles = (n + kTile - 1) / kTile;
    const unsigned grid = (unsigned)(tiles < 148 ? tiles : 148);
    mlp_train_kernel<<<grid, 128, kTrSmem, s>>>(tr->w, x_device, y_device, n, 1.f / (float)n, tr->g, tr->loss,
                                                tr->err);
    ++tr->t;
    const float c1 = 1.f - powf(0.9f, (float)tr->t), c2 = 1.f - powf(0.999f, (float)tr->t);
    adam_kernel<<<(kTrainable + 255) / 256, 256, 0, s>>>(tr->w, tr->g, tr->m, tr->v, kTrainable, lr, c1, c2);
    tr->last_n = n;
    return cudaGetLastError() == cudaSuccess ? ZL_OK : ZL_EDEVICE;
}

static int trainer_check(zl_trainer* tr) {
    if (cudaSetDevice(tr->device) != cudaSuccess || cudaStreamSynchronize(tr->stream) != cudaSuccess)
        return ZL_EDEVICE;
    int e = 0;
    if (cudaMemcpy(&e, tr->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return ZL_EDEVICE;
    return e ? ZL_ETIMEOUT : ZL_OK;
}

int zl_trainer_loss(zl_trainer* tr, double* loss) {
    if (!tr || !loss) return ZL_EINVAL;
    int rc = trainer_check(tr);
    if (rc) return rc;
    float v = 0.f;
    if (cudaMemcpy(&v, tr->loss, sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) return ZL_EDEVICE;
    *loss = tr->last_n > 0 ? (double)v / (double)tr->last_n : 0.;
    return ZL_OK;
}

int zl_trainer_gradients(zl_trainer* tr, zl_mlp* grad) {
    if (!tr || !grad) return ZL_EINVAL;
    int rc = trainer_check(tr);
    if (rc) return rc;
    std::memset(grad, 0, sizeof(zl_mlp));
    return cudaMemcpy(grad, tr->g, sizeof(float) * kTrainable, cudaMemcpyDeviceToHost) == cudaSuccess ? ZL_OK
                                                                                                      : ZL_EDEVICE;
}

int zl_trainer_weights(zl_trainer* tr, zl_mlp* out) {
    if (!tr || !out) return ZL_EINVAL;
    int rc = trainer_check(tr);
    if (rc) return rc;
    return cudaMemcpy(out, tr->w, sizeof(zl_mlp), cudaMemcpyDeviceToHost) == cudaSuccess ? ZL_OK : ZL_EDEVICE;
}

void zl_trainer_destroy(zl_trainer* tr) {
    if (!tr) return;
    cudaSetDevice(tr->device);
    if (tr->stream) cudaStreamSynchronize(tr->stream);
    if (tr->own_stream && tr->own_stream != tr->stream) cudaStreamSynchronize(tr->own_stream);
    cudaFree(tr->w);
    cudaFree(tr->g);
    cudaFree(tr->m);
    cudaFree(tr->v);
    cudaFree(tr->loss);
    cudaFree(tr->err);
    if (tr->own_stream) cudaStreamDestroy(tr->own_stream);
    delete tr;
}

int zl_mlp_forward(const zl_mlp* net, const float* x_device, int64_t n, float* y_device, void* stream) {
    if (!net || !x_device || !y_device || n < 0) return ZL_EINVAL;
    if (n == 0) return ZL_OK;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return ZL_EDEVICE;
    int rc = train_attr_once(device);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float* w = nullptr;
    int* err = nullptr;
    if (cudaMalloc(&w, sizeof(zl_mlp)) != cudaSuccess || cudaMalloc(&err, sizeof(int)) != cudaSuccess) {
        cudaFree(w);
        return ZL_EDEVICE;
    }
    int e = 0;
    bool ok = cudaMemcpyAsync(w, net, sizeof(zl_mlp), cudaMemcpyHostToDevice, s) == cudaSuccess &&
              cudaMemsetAsync(err, 0, sizeof(int), s) == cudaSuccess;
    if (ok) {
        const long long tiles = (n + kTile - 1) / kTile;
        const long long cap = 148 * 4;  // four CTAs per SM: 4 x 64 TMEM columns and 4 x 37 KiB
        const unsigned grid = (unsigned)(tiles < cap ? tiles : cap);
        mlp_forward_kernel<<<grid, 128, kFwSmemLaunch, s>>>(w, x_device, n, y_device, err);
        ok = cudaGetLastError() == cudaSuccess &&
             cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
             cudaStreamSynchronize(s) == cudaSuccess;
    }
    cudaFree(w);
    cudaFree(err);
    if (!ok) return ZL_EDEVICE;
    return e ? ZL_ETIMEOUT : ZL_OK;
}

int zl_closure_pairs(const int32_t nc[3], const float* filtered_device, double tau_fine, double tau_coarse,
                     int factor, float* x_device, float* y_device, float* scratch_device, void* stream) {
    if (!nc || !filtered_device || !x_device || !y_device || !scratch_device || factor < 1 || !(tau_fine > 0.5) ||
        !(tau_coarse > 0.5))
        return ZL_EINVAL;
    Grid3 g;
    for (int a = 0; a < 3; ++a) {
        if (nc[a] < 3) return ZL_EINVAL;
        g.n[a] = nc[a];
    }
    const long long nn = (long long)nc[0] * nc[1] * nc[2];
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const unsigned blocks = (unsigned)((nn + 255) / 256);
    pairs_stage1_kernel<<<blocks, 256, 0, s>>>(g, filtered_device, (float)tau_fine, factor, scratch_device);
    pairs_stage2_kernel<<<blocks, 256, 0, s>>>(g, filtered_device, scratch_device, (float)tau_fine, (float)tau_coarse,
                                               factor, x_device, y_device);
    return cudaGetLastError() == cudaSuccess ? ZL_OK : ZL_EDEVICE;
}

}  // extern "C"
