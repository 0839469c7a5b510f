// Fifth-generation tensor-core (tcgen05) primitives for sm_100a: shared-memory matrix
// descriptors, BF16 x BF16 -> FP32 MMA with the accumulator in tensor memory (TMEM), TMEM
// allocation and loads, mbarrier completion with bounded waits.
//
// Operand tiles live in shared memory without swizzle as 8 x 16-byte core matrices:
//     element (r, k) of a tile with row stride group `sbo` bytes sits at
//     (r / 8) * sbo + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.
// Read with k as the reduction index the tile is "K-major"; read with r as the reduction index
// the same bytes form an "MN-major" operand (its 8-element rows are contiguous along M or N).
// So one buffer serves as A of X W^T and, transposed, as an operand of the weight gradient.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace zl {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (r, k) in a tile whose 8-row groups are `sbo` bytes apart
__host__ __device__ constexpr uint32_t tile_offset(uint32_t r, uint32_t k, uint32_t sbo) {
    return (r >> 3) * sbo + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor (no swizzle): start address, leading-dimension byte offset
// (between the two 8-element core matrices of one K = 16 slice) and stride-dimension byte offset
// (between 8-row groups along M or N); bits 46-47 = 1 select the sm_100 descriptor format.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// K-major operand of a K = 16 slice s of a tile with row-group stride sbo
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t base, uint32_t sbo, int s) {
    return sdesc(base + 256u * (uint32_t)s, 128u, sbo);
}
// MN-major operand: the tile's rows are the reduction index; slice s covers rows 16 s .. 16 s + 15
__device__ __forceinline__ uint64_t desc_mnmajor(uint32_t base, uint32_t sbo, int s) {
    return sdesc(base + 2u * sbo * (uint32_t)s, sbo, 128u);
}

// last byte + 1 that a descriptor reads, for compile-time bounds checks of the tile buffers
__host__ __device__ constexpr uint32_t extent_kmajor(uint32_t rows, uint32_t sbo, int slices) {
    return 256u * (uint32_t)(slices - 1) + (rows / 8 - 1) * sbo + 128u + 128u;
}
__host__ __device__ constexpr uint32_t extent_mnmajor(uint32_t cols, uint32_t sbo, int slices) {
    return (2u * (uint32_t)(slices - 1) + 1u) * sbo + (cols / 8 - 1) * 128u + 128u;
}

// Instruction descriptor of kind::f16 with BF16 A and B and an FP32 accumulator
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n, bool a_mn_major, bool b_mn_major) {
    return (1u << 4)                         // D format F32
           | (1u << 7) | (1u << 10)          // A, B format BF16
           | ((a_mn_major ? 1u : 0u) << 15) | ((b_mn_major ? 1u : 0u) << 16)
           | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D[tmem] (+)= A * B^T, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate ? 1u : 0u));
}

// arrive on the mbarrier once every MMA this thread issued before has completed
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity to complete; false when `limit` polls ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// whole warp: allocate ncols TMEM columns (a power of two >= 32), address written to *dst
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// make generic-proxy shared-memory writes visible to the tensor cores
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Warp-collective: lane t of the warp reads TMEM lane (taddr lane + t), 16 consecutive columns.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 8 BF16 values packed for one 16-byte core-matrix row
__device__ __forceinline__ uint4 pack_bf16x8(const float* v) {
    uint4 o;
    __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]),
                   c = __floats2bfloat162_rn(v[4], v[5]), d = __floats2bfloat162_rn(v[6], v[7]);
    o.x = *reinterpret_cast<uint32_t*>(&a);
    o.y = *reinterpret_cast<uint32_t*>(&b);
    o.z = *reinterpret_cast<uint32_t*>(&c);
    o.w = *reinterpret_cast<uint32_t*>(&d);
    return o;
}

}  // namespace tc
}  // namespace zl
