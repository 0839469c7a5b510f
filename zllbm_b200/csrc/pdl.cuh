// Programmatic dependent launch (sm_90 and later): a kernel launched with launch_dependent may be
// scheduled while the kernel before it on the stream is still running; it waits in pdl_wait()
// until that kernel has finished and its writes are visible, so only its launch and block
// scheduling overlap the previous kernel's tail.  The per-step kernels of small levels (a few
// thousand nodes: immersed-boundary passes, transfers, face passes, fine-level steps) are chains
// of short dependent launches, where that latency is most of the time.
//
// Every kernel launched with launch_dependent calls pdl_wait() before it reads or writes global
// memory; pdl_trigger() lets the next kernel's launch begin once every block of this one has
// started (a kernel that never calls it triggers when it exits).  In a kernel not launched with
// launch_dependent both are no-ops.
#pragma once
#include <cuda_runtime.h>
#include <utility>

namespace zl {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <class... KernelArgs, class... Args>
cudaError_t launch_dependent(void (*kernel)(KernelArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                             Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace zl

// Dependent launch inside a function returning cudaError_t: returns the launch error, if any.
#define ZL_LAUNCH_DEP(...)                                                          \
    do {                                                                            \
        const cudaError_t zl_launch_err_ = ::zl::launch_dependent(__VA_ARGS__);     \
        if (zl_launch_err_ != cudaSuccess) return zl_launch_err_;                   \
    } while (0)
