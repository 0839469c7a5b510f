// Launchers of the fused step (one parity of the AA pattern) and of the batched multi-level
// step (one set of extensions) for one (storage, lattice, collision).  Only step_inst.cu includes this file: it is
// compiled once per combination, each with an explicit instantiation, so the build compiles the
// step kernel variants in parallel translation units.  The launch sets of launch.cuh call them
// through the declarations there.
#pragma once
#include "launch.cuh"

namespace zl {
namespace step_impl {

// D3Q19 with the default block shape and rows whose length is not a multiple of 32: the threads
// are numbered over each x-y plane (no warp holds the few nodes left at a row's end on its own),
// rows' end nodes last when the x axis is bounded; a level of a few thousand nodes takes one-warp
// blocks, so that its launch still reaches every SM.
// (Measured: the flow past a cube 3 % faster; D2Q9 levels are faster per row, 3 % on the
// cylinder flow.)
template <class S, class L, int C, bool O, bool B, bool M, int X = 0>
cudaError_t step_one(S* f, const LevelGeom& geo, const StepParams& p, cudaStream_t s) {
    dim3 g, b;
    step_shape(geo, L::kDims, g, b);
    const bool default_shape = geo.block[0] == 0 || geo.block[0] == kRowKernelBlockX;
    const long long plane = (long long)geo.n[0] * geo.n[1];
    if (L::kDims == 3 && default_shape && (geo.n[0] & 31) && plane < (1ll << 31)) {
        LevelGeom fg = geo;
        // a non-periodic x axis: every row's two end nodes patch missing upstream values, and
        // numbered in row order they would put the patch path into most warps of a plane; the
        // threads take the rows' inner nodes first and the end nodes last (a few warps per plane)
        const bool ends_last = (B || M) && !geo.periodic[0] && geo.n[0] >= 3;
        fg.flat = ends_last ? 2 : 1;
        fg.fn0 = FastDiv::make((uint32_t)(ends_last ? geo.n[0] - 2 : geo.n[0]));
        const unsigned bs = plane * g.z >= 148ll * 128 * 8 ? 128u : 32u;
        ZL_LAUNCH_DEP(aa_step_kernel<L, S, C, O, B, M, X>, dim3((unsigned)((plane + bs - 1) / bs), 1, g.z), dim3(bs), 0, s,
                      f, fg, p);
        return cudaGetLastError();
    }
    ZL_LAUNCH_DEP(aa_step_kernel<L, S, C, O, B, M, X>, g, b, 0, s, f, geo, p);
    return cudaGetLastError();
}

template <class S, int C, bool O>
cudaError_t step_pair(S* f, const LevelGeom& geo, const StepParams& p, cudaStream_t s) {
    if constexpr (Storage<S>::kDeviation) {
        if ((geo.n[0] & 1) || (geo.stride & 1)) {
            // pair accesses need an even row length and plane stride: scalar kernel instead
            LevelGeom g1 = geo;
            g1.block[0] = g1.block[1] = 0;
            return step_one<S, D3Q19, C, O, false, false>(f, g1, p, s);
        }
        dim3 g, b;
        step_shape(geo, 3, g, b);
        ZL_LAUNCH_DEP(aa_pair_kernel<S, C, O>, g, b, 0, s, f, geo, p);
        return cudaGetLastError();
    }
    return cudaErrorInvalidValue;
}

template <class S, int C, bool O>
cudaError_t step_row(S* f, const LevelGeom& geo, const StepParams& p, cudaStream_t s) {
    if constexpr (sizeof(S) == 2) {
        const int v = row_kernel_width(geo);
        const int rows = geo.block[1];
        if (v == 0 || rows < 1 || rows > 4) return cudaErrorInvalidValue;
        const dim3 b(32 * rows), g((geo.n[1] + rows - 1) / rows, geo.zn > 0 ? geo.zn : geo.n[2]);
        if (v == 8) ZL_LAUNCH_DEP(aa_row_kernel<S, C, O, 8>, g, b, 0, s, f, geo, p);
        else ZL_LAUNCH_DEP(aa_row_kernel<S, C, O, 4>, g, b, 0, s, f, geo, p);
        return cudaGetLastError();
    }
    return cudaErrorInvalidValue;
}

}  // namespace step_impl

template <class S, class L, int C, bool O>
cudaError_t step_lco(bool bnd, bool masked, S* f, const LevelGeom& geo, const StepParams& p, cudaStream_t s) {
    using namespace step_impl;
    if constexpr (L::kDims == 3) {
        if (geo.block[0] == kRowKernelBlockX && row_eligible(3, bnd, masked, p, (int)sizeof(S), geo))
            return step_row<S, C, O>(f, geo, p, s);
        if (geo.block[0] < 0 && pair_eligible(3, bnd, masked, p, (int)sizeof(S), geo))
            return step_pair<S, C, O>(f, geo, p, s);
    }
    if (p.forced || p.les) {
        if (!masked) return cudaErrorInvalidValue;
        if (p.forced && p.les) return step_one<S, L, C, O, true, true, kExtForce | kExtLes>(f, geo, p, s);
        if (p.forced) return step_one<S, L, C, O, true, true, kExtForce>(f, geo, p, s);
        return step_one<S, L, C, O, true, true, kExtLes>(f, geo, p, s);
    }
    if (masked) return step_one<S, L, C, O, true, true>(f, geo, p, s);
    if (bnd) return step_one<S, L, C, O, true, false>(f, geo, p, s);
    return step_one<S, L, C, O, false, false>(f, geo, p, s);
}

template <class S, class L, int C, int X>
cudaError_t batch_lcx(const LevelBatch& b, cudaStream_t s) {
    const long long total = b.first[b.count];
    if (total <= 0) return cudaSuccess;
    const long long want = (total + kBatchThreads - 1) / kBatchThreads, cap = 148 * 6;
    const unsigned blocks = (unsigned)(want < cap ? want : cap);
    aa_batch_kernel<L, S, C, X><<<blocks, kBatchThreads, 0, s>>>(b);
    return cudaGetLastError();
}

}  // namespace zl
