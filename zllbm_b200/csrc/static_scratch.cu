// zl_moments_noalloc: FP64 mass and momentum sums over a caller-owned population array,
// with no device allocation.
//
// This is the allocation-free twin of the conservation reduction behind zl_conservation.
// It exists for callers that cannot call cudaMalloc: code issuing work from a loop where a
// cudaMalloc / cudaFree would synchronize the whole device, a host whose device memory is
// entirely handed out by another allocator (a framework's memory pool), or code that must
// not fail on allocation once it is running.  Such a caller passes its own device arrays for
// the input populations and the output sums; the per-block partial sums live in the
// file-scope array below, which every GPU that loads the library holds until process exit.
#include <cuda_runtime.h>
#include <mutex>
#include "zllbm_b200.h"
#include "lattice.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 4096;          // partial sums held by the static scratch
constexpr long long kNodesPerBlock = 4096;  // nodes reduced by one block
constexpr long long kMaxNodes = kMaxBlocks * kNodesPerBlock;  // 16,777,216 nodes per call
constexpr int kMaxDevices = 64;

}  // namespace

// Block partials: kMaxBlocks x {mass, jx, jy, jz}, 128 KiB per device.
static __device__ __align__(256) double g_moment_scratch[kMaxBlocks * 4];

namespace {

// Per-block partial sums of rho, jx, jy, jz over kNodesPerBlock nodes; the direction tables
// are compile-time constants of the lattice (reference direction order), folded after unrolling.
template <class L>
__global__ void __launch_bounds__(kThreads) moments_partial_static(const double* __restrict__ f, long long n,
                                                                   double* __restrict__ partial) {
    using Tb = zl::Tables<L>;
    constexpr int Q = L::kQ;
    __shared__ double red[4][kThreads / 32];
    const long long first = (long long)blockIdx.x * kNodesPerBlock;
    const long long last = first + kNodesPerBlock < n ? first + kNodesPerBlock : n;
    double acc[4] = {0., 0., 0., 0.};
    for (long long i = first + threadIdx.x; i < last; i += kThreads) {
        const double* node = f + i * Q;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            const double v = node[k];
            acc[0] += v;
            if (Tb::cx(k)) acc[1] += Tb::cx(k) > 0 ? v : -v;
            if (Tb::cy(k)) acc[2] += Tb::cy(k) > 0 ? v : -v;
            if (Tb::cz(k)) acc[3] += Tb::cz(k) > 0 ? v : -v;
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
        for (int w = 0; w < kThreads / 32; ++w) v += red[threadIdx.x][w];
        partial[blockIdx.x * 4 + threadIdx.x] = v;  // every launched block writes its slot
    }
}

__global__ void moments_final_static(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
    if (threadIdx.x < 4) {
        double v = 0.;
        for (int b = 0; b < nblocks; ++b) v += partial[b * 4 + threadIdx.x];
        out[threadIdx.x] = v;
    }
}

std::mutex g_mutex;
double* g_scratch[kMaxDevices] = {};

// Device address of the static scratch on the current device.  In host code the name
// g_moment_scratch only stands for the symbol; the address a kernel may use comes from
// cudaGetSymbolAddress, looked up once per device with that device current.
int scratch_address(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return ZL_EDEVICE;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch[dev]) {
        void* addr = nullptr;
        if (cudaGetSymbolAddress(&addr, g_moment_scratch) != cudaSuccess || !addr) return ZL_EDEVICE;
        g_scratch[dev] = static_cast<double*>(addr);
    }
    *out = g_scratch[dev];
    return ZL_OK;
}

}  // namespace

extern "C" int zl_moments_noalloc(int lattice, const double* f_device, int64_t n, double* out_device,
                                  void* stream) {
    if (lattice != ZL_D2Q9 && lattice != ZL_D3Q19) return ZL_EINVAL;
    if (!f_device || !out_device || n <= 0) return ZL_EINVAL;
    if (n > kMaxNodes) return ZL_ETOOLARGE;
    double* partial = nullptr;
    const int rc = scratch_address(&partial);
    if (rc != ZL_OK) return rc;
    const int blocks = (int)((n + kNodesPerBlock - 1) / kNodesPerBlock);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // cudaLaunchKernel returns the status of this launch only; the runtime's last-error slot,
    // which may hold an earlier unrelated failure of the caller, is neither read nor cleared.
    const void* partial_fn = lattice == ZL_D2Q9 ? (const void*)moments_partial_static<zl::D2Q9>
                                                 : (const void*)moments_partial_static<zl::D3Q19>;
    long long nn = n;
    void* partial_args[] = {(void*)&f_device, (void*)&nn, (void*)&partial};
    if (cudaLaunchKernel(partial_fn, dim3(blocks), dim3(kThreads), partial_args, 0, s) != cudaSuccess)
        return ZL_EDEVICE;
    const double* partial_in = partial;
    int nb = blocks;
    void* final_args[] = {(void*)&partial_in, (void*)&nb, (void*)&out_device};
    if (cudaLaunchKernel((const void*)moments_final_static, dim3(1), dim3(32), final_args, 0, s) != cudaSuccess)
        return ZL_EDEVICE;
    return ZL_OK;
}
