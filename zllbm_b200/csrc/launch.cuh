// Host-side launchers for one population storage type.  Each storage type is
// compiled in its own translation unit (the FP64 one with -fmad=false, so its
// arithmetic follows the reference's rounding step for step).
#pragma once
#include <cuda_runtime.h>
#include "ib.cuh"
#include "row_kernel.cuh"

namespace zl {

struct LaunchSet {
    int elem_bytes;
    cudaError_t (*step)(int dims, int coll, bool odd, bool bnd, bool masked, void* f, const LevelGeom& geo,
                        const StepParams& p, cudaStream_t s);
    cudaError_t (*neq)(int dims, void* f, const LevelGeom& geo, const StepParams& p, int face, int even_layout,
                       const double* feq_b, cudaStream_t s);
    // kind: ZL_BC_BOUNCE_BACK, ZL_BC_PERIODIC or ZL_BC_CONVECTIVE_OUTFLOW face pass
    cudaError_t (*face)(int dims, int kind, void* f, const LevelGeom& geo, const StepParams& p, int face,
                        int even_layout, cudaStream_t s);
    cudaError_t (*scatter)(int dims, void* f, const LevelGeom& geo, const StepParams& p, const LevelMap& m,
                           int even_layout, const uint64_t* codes, const double* fin, long long n, int* bad,
                           cudaStream_t s);
    cudaError_t (*gather)(int dims, const void* f, const LevelGeom& geo, const StepParams& p, const LevelMap& m,
                          int even_layout, const uint64_t* codes, double* fout, double* rho, double* u, long long n,
                          int* bad, cudaStream_t s);
    cudaError_t (*conservation)(int dims, const void* f, const LevelGeom& geo, const StepParams& p,
                                int even_layout, double* partial, int nblocks, double* out, cudaStream_t s);
    // explosion (save / prev in the storage's arithmetic type); with `with_f2c` (no target a
    // coalescence source) the coalescence too, in the same launch
    cudaError_t (*c2f)(int dims, void* ff, const LevelGeom& fgeo, int f_even, void* fc, const LevelGeom& cgeo,
                       int c_even, const StepParams& fp, const StepParams& cp, const C2FStencil& st, double tau_ratio,
                       void* save, const void* prev, int store, const F2CJob* with_f2c, cudaStream_t s);
    cudaError_t (*f2c)(int dims, const void* ff, const LevelGeom& fgeo, int f_even, void* fc, const LevelGeom& cgeo,
                       int c_even, const StepParams& fp, const StepParams& cp, const F2CJob& job, cudaStream_t s);
    cudaError_t (*ib_touch)(int dims, const void* f, const LevelGeom& geo, const StepParams& p, int even_layout,
                            const int* nodes, int n_nodes, double* node_vel, cudaStream_t s);
    // ext: kExtForce / kExtLes bits of the levels in the batch
    cudaError_t (*batch)(int dims, int coll, int ext, const LevelBatch& b, cudaStream_t s);
};

const LaunchSet& launch_set_f64();
const LaunchSet& launch_set_f32();
const LaunchSet& launch_set_f16();
const LaunchSet& launch_set_bf16();

// Block shape and grid of the fused step: one thread per node, x fastest.  The shape is the
// level's autotuned choice (zl_autotune) or a default of up to 128 threads along x.
// A negative block x selects the two-nodes-per-thread kernel with |x| threads along x.
inline void step_shape(const LevelGeom& geo, int dims, dim3& grid, dim3& block) {
    int bx = geo.block[0], by = geo.block[1];
    int nx = geo.n[0];
    if (bx == kRowKernelBlockX) bx = by = 0;  // row-kernel choice: other kernels take the default shape
    if (bx < 0) {
        bx = -bx;
        nx = (nx + 1) / 2;
    }
    if (bx <= 0 || by <= 0) {
        bx = 128;  // measured faster than 256 for the D3Q19 step on B200 (more CTAs in flight per SM)
        while (bx > 32 && bx / 2 >= nx) bx /= 2;
        by = 1;
    }
    block = dim3(bx, by, 1);
    grid = dim3((nx + bx - 1) / bx, (geo.n[1] + by - 1) / by, dims == 3 ? (geo.zn > 0 ? geo.zn : geo.n[2]) : 1);
}

// The two-nodes-per-thread kernel applies to full periodic D3Q19 boxes (or slabs of one, geo.ring)
// in deviation storage without forcing or LES.
inline bool pair_eligible(int dims, bool bnd, bool masked, const StepParams& p, int elem_bytes,
                          const LevelGeom& geo) {
    return dims == 3 && (geo.ring || (!bnd && !masked)) && !p.forced && !p.les && elem_bytes < 8;
}

// The one-warp-per-row kernel (row_kernel.cuh): full periodic D3Q19 boxes in 16-bit storage
// with rows of 128 or 256 nodes, no forcing or LES.
inline bool row_eligible(int dims, bool bnd, bool masked, const StepParams& p, int elem_bytes,
                         const LevelGeom& geo) {
    return pair_eligible(dims, bnd, masked, p, elem_bytes, geo) && elem_bytes == 2 && row_kernel_width(geo) != 0;
}

// Fused step launchers of one (storage, lattice, collision, parity) and batched step launchers
// of one (storage, lattice, collision, extensions), defined in step_launch.cuh and instantiated
// in step_inst.cu (one translation unit per combination).
template <class S, class L, int C, bool O>
cudaError_t step_lco(bool bnd, bool masked, S* f, const LevelGeom& geo, const StepParams& p, cudaStream_t s);
template <class S, class L, int C, int X>
cudaError_t batch_lcx(const LevelBatch& b, cudaStream_t s);
template <class S, class L, int C>
cudaError_t batch_lc(int ext, const LevelBatch& b, cudaStream_t s) {
    switch (ext) {
        case 0: return batch_lcx<S, L, C, 0>(b, s);
        case kExtForce: return batch_lcx<S, L, C, kExtForce>(b, s);
        case kExtLes: return batch_lcx<S, L, C, kExtLes>(b, s);
        default: return batch_lcx<S, L, C, kExtForce | kExtLes>(b, s);
    }
}
template <class S, class L, int C>
cudaError_t step_lc(bool odd, bool bnd, bool masked, S* f, const LevelGeom& geo, const StepParams& p,
                    cudaStream_t s) {
    return odd ? step_lco<S, L, C, true>(bnd, masked, f, geo, p, s) : step_lco<S, L, C, false>(bnd, masked, f, geo, p, s);
}

#define ZL_DEFINE_LAUNCH_SET(NAME, S)                                                                            \
    namespace NAME##_impl {                                                                                      \
    cudaError_t step_any(int dims, int coll, bool odd, bool bnd, bool masked, void* fv, const LevelGeom& geo,    \
                         const StepParams& p, cudaStream_t s) {                                                  \
        S* f = static_cast<S*>(fv);                                                                              \
        if (dims == 2)                                                                                           \
            return coll == kMrt ? step_lc<S, D2Q9, kMrt>(odd, bnd, masked, f, geo, p, s)                            \
                                : step_lc<S, D2Q9, kSrt>(odd, bnd, masked, f, geo, p, s);                           \
        return coll == kMrt ? step_lc<S, D3Q19, kMrt>(odd, bnd, masked, f, geo, p, s)                               \
                            : step_lc<S, D3Q19, kSrt>(odd, bnd, masked, f, geo, p, s);                              \
    }                                                                                                            \
    cudaError_t neq_any(int dims, void* fv, const LevelGeom& geo, const StepParams& p, int face, int even,       \
                        const double* feq_b, cudaStream_t s) {                                                   \
        S* f = static_cast<S*>(fv);                                                                              \
        const int axis = face >> 1;                                                                              \
        const int o0 = axis == 0 ? 1 : 0, o1 = axis == 2 ? 1 : 2;                                                \
        const int n0 = geo.n[o0], n1 = dims == 3 ? geo.n[o1] : 1;                                                \
        dim3 b(128), g((n0 + 127) / 128, n1);                                                                    \
        if (dims == 2)                                                                                           \
            ZL_LAUNCH_DEP(neq_face_kernel<D2Q9, S>, g, b, 0, s, f, geo, p, face, even, feq_b);                              \
        else                                                                                                     \
            ZL_LAUNCH_DEP(neq_face_kernel<D3Q19, S>, g, b, 0, s, f, geo, p, face, even, feq_b);                             \
        return cudaGetLastError();                                                                               \
    }                                                                                                            \
    cudaError_t face_any(int dims, int kind, void* fv, const LevelGeom& geo, const StepParams& p, int face,     \
                         int even, cudaStream_t s) {                                                             \
        S* f = static_cast<S*>(fv);                                                                              \
        const int axis = face >> 1;                                                                              \
        const int o0 = axis == 0 ? 1 : 0, o1 = axis == 2 ? 1 : 2;                                                \
        const int n0 = geo.n[o0], n1 = dims == 3 ? geo.n[o1] : 1;                                                \
        dim3 b(128), g((n0 + 127) / 128, n1);                                                                    \
        if (dims == 2) {                                                                                         \
            if (kind == kBcBounceBack) ZL_LAUNCH_DEP(bb_face_kernel<D2Q9, S>, g, b, 0, s, f, geo, p, face, even);           \
            else if (kind == kBcConvective) ZL_LAUNCH_DEP(conv_face_kernel<D2Q9, S>, g, b, 0, s, f, geo, p, face, even);    \
            else ZL_LAUNCH_DEP(periodic_face_kernel<D2Q9, S>, g, b, 0, s, f, geo, p, face, even);                           \
        } else {                                                                                                 \
            if (kind == kBcBounceBack) ZL_LAUNCH_DEP(bb_face_kernel<D3Q19, S>, g, b, 0, s, f, geo, p, face, even);          \
            else if (kind == kBcConvective) ZL_LAUNCH_DEP(conv_face_kernel<D3Q19, S>, g, b, 0, s, f, geo, p, face, even);   \
            else ZL_LAUNCH_DEP(periodic_face_kernel<D3Q19, S>, g, b, 0, s, f, geo, p, face, even);                          \
        }                                                                                                        \
        return cudaGetLastError();                                                                               \
    }                                                                                                            \
    cudaError_t scatter_any(int dims, void* fv, const LevelGeom& geo, const StepParams& p, const LevelMap& m,    \
                            int even, const uint64_t* codes, const double* fin, long long n, int* bad,           \
                            cudaStream_t s) {                                                                    \
        if (n <= 0) return cudaSuccess;                                                                          \
        S* f = static_cast<S*>(fv);                                                                              \
        const unsigned blocks = (unsigned)((n + 255) / 256);                                                     \
        if (dims == 2)                                                                                           \
            scatter_kernel<D2Q9, S><<<blocks, 256, 0, s>>>(f, geo, p, m, even, codes, fin, n, bad);              \
        else                                                                                                     \
            scatter_kernel<D3Q19, S><<<blocks, 256, 0, s>>>(f, geo, p, m, even, codes, fin, n, bad);             \
        return cudaGetLastError();                                                                               \
    }                                                                                                            \
    cudaError_t gather_any(int dims, const void* fv, const LevelGeom& geo, const StepParams& p,                  \
                           const LevelMap& m, int even, const uint64_t* codes, double* fout, double* rho,        \
                           double* u, long long n, int* bad, cudaStream_t s) {                                   \
        if (n <= 0) return cudaSuccess;                                                                          \
        const S* f = static_cast<const S*>(fv);                                                                  \
        const unsigned blocks = (unsigned)((n + 255) / 256);                                                     \
        if (dims == 2)                                                                                           \
            gather_kernel<D2Q9, S><<<blocks, 256, 0, s>>>(f, geo, p, m, even, codes, fout, rho, u, n, bad);        \
        else                                                                                                     \
            gather_kernel<D3Q19, S><<<blocks, 256, 0, s>>>(f, geo, p, m, even, codes, fout, rho, u, n, bad);       \
        return cudaGetLastError();                                                                               \
    }                                                                                                            \
    cudaError_t conservation_any(int dims, const void* fv, const LevelGeom& geo, const StepParams& p, int even,  \
                                 double* partial, int nblocks, double* out, cudaStream_t s) {                    \
        const S* f = static_cast<const S*>(fv);                                                                  \
        if (dims == 2)                                                                                           \
            conservation_partial_kernel<D2Q9, S><<<nblocks, 256, 0, s>>>(f, geo, p, even, partial);              \
        else                                                                                                     \
            conservation_partial_kernel<D3Q19, S><<<nblocks, 256, 0, s>>>(f, geo, p, even, partial);             \
        cudaError_t e = cudaGetLastError();                                                                      \
        if (e != cudaSuccess) return e;                                                                          \
        conservation_final_kernel<<<1, 32, 0, s>>>(partial, nblocks, out);                                       \
        return cudaGetLastError();                                                                               \
    }                                                                                                            \
    cudaError_t c2f_any(int dims, void* ff, const LevelGeom& fgeo, int f_even, void* fc, const LevelGeom& cgeo,     \
                        int c_even, const StepParams& fp, const StepParams& cp, const C2FStencil& st,            \
                        double tau_ratio, void* save, const void* prev, int store, const F2CJob* with_f2c,       \
                        cudaStream_t s) {                                                                        \
        if (st.n_targets <= 0) return cudaSuccess;                                                               \
        using T = typename Storage<S>::T;                                                                        \
        const int q = dims == 2 ? 9 : 19;                                                                        \
        const unsigned sblocks = (unsigned)((st.n_sources + 127) / 128);                                         \
        const int lanes = sizeof(T) == 8 ? q : (q + 3) / 4; /* threads per target (c2f_lanes) */                 \
        const unsigned wblocks = (unsigned)(((long long)st.n_targets * lanes + kC2fThreads - 1) / kC2fThreads); \
        const unsigned fblocks = with_f2c ? (unsigned)(((long long)with_f2c->n * q + kC2fThreads - 1) /          \
                                                       kC2fThreads) : 0u;                                        \
        if (dims == 2) {                                                                                         \
            if (st.n_sources > 0)                                                                                \
                ZL_LAUNCH_DEP(c2f_sources_kernel<D2Q9, S>, sblocks, 128, 0, s, (const S*)ff, fgeo, f_even, (const S*)fc,    \
                                                                    cgeo, c_even, fp, cp, st, tau_ratio);        \
            if (with_f2c)                                                                                        \
                ZL_LAUNCH_DEP(c2f_f2c_kernel<D2Q9, S>, wblocks + fblocks, kC2fThreads, 0, s,                                \
                    (S*)ff, fgeo, f_even, fp, st, (T*)save, (S*)fc, cgeo, c_even, cp, *with_f2c, wblocks);       \
            else                                                                                                 \
                ZL_LAUNCH_DEP(c2f_kernel<D2Q9, S>, wblocks, kC2fThreads, 0, s, (S*)ff, fgeo, f_even, fp, st, (T*)save,      \
                                                                     (const T*)prev, store);                     \
        } else {                                                                                                 \
            if (st.n_sources > 0)                                                                                \
                ZL_LAUNCH_DEP(c2f_sources_kernel<D3Q19, S>, sblocks, 128, 0, s, (const S*)ff, fgeo, f_even, (const S*)fc,   \
                                                                     cgeo, c_even, fp, cp, st, tau_ratio);       \
            if (with_f2c)                                                                                        \
                ZL_LAUNCH_DEP(c2f_f2c_kernel<D3Q19, S>, wblocks + fblocks, kC2fThreads, 0, s,                               \
                    (S*)ff, fgeo, f_even, fp, st, (T*)save, (S*)fc, cgeo, c_even, cp, *with_f2c, wblocks);       \
            else                                                                                                 \
                ZL_LAUNCH_DEP(c2f_kernel<D3Q19, S>, wblocks, kC2fThreads, 0, s, (S*)ff, fgeo, f_even, fp, st, (T*)save,     \
                                                                      (const T*)prev, store);                    \
        }                                                                                                        \
        return cudaGetLastError();                                                                               \
    }                                                                                                            \
    cudaError_t f2c_any(int dims, const void* ff, const LevelGeom& fgeo, int f_even, void* fc,                   \
                        const LevelGeom& cgeo, int c_even, const StepParams& fp, const StepParams& cp,           \
                        const F2CJob& job, cudaStream_t s) {                                                     \
        if (job.n <= 0) return cudaSuccess;                                                                      \
        /* one thread per (node, population), 64-thread blocks spread them over every SM */                     \
        const unsigned blocks = (unsigned)(((long long)job.n * (dims == 2 ? 9 : 19) + 63) / 64);                 \
        if (dims == 2)                                                                                           \
            ZL_LAUNCH_DEP(f2c_kernel<D2Q9, S>, blocks, 64, 0, s, (const S*)ff, fgeo, f_even, (S*)fc, cgeo, c_even, fp, cp,  \
                                                      job);                                                      \
        else                                                                                                     \
            ZL_LAUNCH_DEP(f2c_kernel<D3Q19, S>, blocks, 64, 0, s, (const S*)ff, fgeo, f_even, (S*)fc, cgeo, c_even, fp, cp, \
                                                       job);                                                     \
        return cudaGetLastError();                                                                               \
    }                                                                                                            \
    cudaError_t ib_touch_any(int dims, const void* f, const LevelGeom& geo, const StepParams& p, int even,      \
                             const int* nodes, int n_nodes, double* node_vel,                                   \
                             cudaStream_t s) {                                                                   \
        if (n_nodes <= 0) return cudaSuccess;                                                                    \
        const unsigned blocks = (unsigned)((n_nodes + 127) / 128);                                               \
        if (dims == 2)                                                                                           \
            ZL_LAUNCH_DEP(ib_touch_kernel<D2Q9, S>, blocks, 128, 0, s, (const S*)f, geo, p, even, nodes, n_nodes,           \
                                                            node_vel);                                           \
        else                                                                                                     \
            ZL_LAUNCH_DEP(ib_touch_kernel<D3Q19, S>, blocks, 128, 0, s, (const S*)f, geo, p, even, nodes, n_nodes,          \
                                                             node_vel);                                          \
        return cudaGetLastError();                                                                               \
    }                                                                                                            \
    cudaError_t batch_any(int dims, int coll, int ext, const LevelBatch& b, cudaStream_t s) {                    \
        if (dims == 2)                                                                                           \
            return coll == kMrt ? batch_lc<S, D2Q9, kMrt>(ext, b, s) : batch_lc<S, D2Q9, kSrt>(ext, b, s);             \
        return coll == kMrt ? batch_lc<S, D3Q19, kMrt>(ext, b, s) : batch_lc<S, D3Q19, kSrt>(ext, b, s);               \
    }                                                                                                            \
    }                                                                                                            \
    const LaunchSet& NAME() {                                                                                    \
        static const LaunchSet set = {(int)sizeof(S), NAME##_impl::step_any, NAME##_impl::neq_any,                \
                                      NAME##_impl::face_any,                                                     \
                                      NAME##_impl::scatter_any, NAME##_impl::gather_any,                         \
                                      NAME##_impl::conservation_any, NAME##_impl::c2f_any,                       \
                                      NAME##_impl::f2c_any, NAME##_impl::ib_touch_any,                           \
                                      NAME##_impl::batch_any};                                                   \
        return set;                                                                                              \
    }

}  // namespace zl
