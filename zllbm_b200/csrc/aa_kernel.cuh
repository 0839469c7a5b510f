// Fused collide + stream for one refinement level, single buffer (AA pattern),
// structure-of-arrays populations in a dense, padded box per level.
//
// Replaces the reference's per-level RunSolverOnGivenGrid (collide every node,
// then pull-stream every node through hash-map lookups,
// lbm_project/lbm_solver_interface.cpp:246-262, d3q19_model/lbm_d3q19_solver.cpp:20-136)
// plus the node-local part of ComputeDomainBoundaryCondition (bounce back,
// lbm_project/boundary_conditions/lbm_bounce_back.cpp:28-91; periodic faces
// become index wrap-around).
//
// State between steps is the reference's post-stream population f_, held in
// one of two layouts that alternate every step:
//   after an even step   f(x, q) lives in slot(x - c_q, opp(q))   (q != 0)
//   after an odd step    f(x, q) lives in slot(x, q)
// Slots of cells that hold no node (the one-cell ghost frame of non-periodic
// axes, or cells a refinement level does not cover) carry the reference's
// "stale" values: where the upstream node x - c_q does not exist the
// reference leaves f_(x, q) unchanged (lbm_d3q19_solver.cpp:31-33); here the
// node writes its own pre-collision value into the slot that holds f(x, q).
#pragma once
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "lattice.cuh"
#include "pdl.cuh"

namespace zl {

enum BcKind : int { kBcNone = 0, kBcBounceBack = 1, kBcPeriodic = 2, kBcNeq = 3, kBcConvective = 4 };
enum Collision : int { kSrt = 0, kMrt = 1 };

// Per-cell information for levels whose node set does not fill its box.
constexpr uint32_t kInfoPresent = 1u << 31;
constexpr uint32_t kInfoSaveMacro = 1u << 30;  // keep rho, u of the last collision (coarse/fine transfer source)
constexpr uint32_t kInfoForce = 1u << 23;  // node force may be non-zero (a stencil node of the immersed boundary)
constexpr int kInfoFaceShift = 24;  // 6 bits: on face xmin..zmax (reference boundary node sets)

// extended-physics bits of the step kernel's Ext template argument
constexpr int kExtForce = 1;
constexpr int kExtLes = 2;

// Division of 31-bit unsigned integers by a fixed divisor through one widening multiply and a
// shift (Granlund and Montgomery, "Division by invariant integers using multiplication", PLDI
// 1994, the round-up method): with l = ceil(log2 d) and m = floor(2^(31 + l) / d) + 1,
// floor(n / d) = floor(n m / 2^(31 + l)) for every 0 <= n < 2^31; m < 2^32 for d >= 2.
struct FastDiv {
    uint32_t d = 1, m = 0, shift = 0;
    ZL_HD static FastDiv make(uint32_t divisor) {
        FastDiv f;
        f.d = divisor;
        if (divisor <= 1) return f;
        uint32_t l = 0;
        while ((1ull << l) < divisor) ++l;
        f.shift = 31 + l;
        f.m = (uint32_t)((1ull << f.shift) / divisor + 1);
        return f;
    }
    ZL_HD uint32_t div(uint32_t n) const {
        return d <= 1 ? n : (uint32_t)(((unsigned long long)n * m) >> shift);
    }
};

struct LevelGeom {
    int n[3];          // nodes per axis (periodic axes hold each plane once)
    int g[3];          // ghost frame width per axis (0 on periodic axes, 1 otherwise)
    int a[3];          // allocated extents, n + 2 g
    int periodic[3];   // wrap-around per axis
    long long stride;  // elements between population planes (>= a0 a1 a2)
    int face_on_box;   // bit f: box edge f lies on domain face f (non-periodic faces only)
    int block[2];      // thread-block shape of the step kernel (x, y); {0, 0}: default
    const uint32_t* info;  // per-cell info (masked levels), nullptr for full boxes
    // 1: a full D3Q19 box, periodic along x and y, whose two z faces are halo faces (a slab of a
    // sharded lattice): every upstream node is present, the z ones in the ghost planes, so the
    // kernels of full periodic boxes apply with z addressed through the ghost frame
    int ring;
    FastDiv fa0, fa1;  // division by a[0] and a[1] (cell index -> box coordinates)
    // D3Q19 step launches: planes [z0, z0 + zn) of the last axis; zn = 0: every plane
    int z0, zn;
    // one-node step launches: 1 = threads numbered over each x-y plane (x fastest) instead of per
    // row, so that rows whose length is not a multiple of 32 share warps; fn0 divides by n[0].
    // 2 = the same with each plane's row-inner nodes (x = 1 .. n[0] - 2) first and the rows' end
    // nodes (x = 0, n[0] - 1) last; fn0 divides by n[0] - 2
    int flat;
    FastDiv fn0;
};

struct StepParams {
    double tau;             // relaxation time at this level
    double rho0;            // default density
    int face_kind[6];       // BcKind per face
    double bb_term[6][19];  // 6 rho0 w_o (c_o . U_face) for outgoing direction o
    const double* mrt64;    // dense M^-1 S M, reference construction order (FP64 mode)
    float mrt_coef[19];     // (s_k - 1/tau) / |M_k|^2 per non-shear moment, 0 elsewhere (fast path)
    float omega32;          // 1/tau in FP32 (fast path)
    float inv_scale;        // reduced storage: deviation = stored * inv_scale
    float scale;
    double scale_d;         // the same scale in FP64 (1 for FP64 / FP32 storage)
    int fuse_bb;            // bounce back applied inside the step kernel (no ordered face passes needed)
    double* macro;          // rho, ux, uy, uz per cell for nodes flagged kInfoSaveMacro (else unused)
    // body forces (Guo forcing): F = const_force + force[cell] (GetAllForcesForANode,
    // lbm_solver_interface.cpp:132-144); force is dims-strided by 3, or nullptr
    const double* force;
    double const_force[3];
    int forced;             // the level collides with forcing (requires the masked layout)
    double dt;              // time step of the level, 2^-level
    const double* mrt64_d;  // dense M^-1 (I - S/2) M (FP64 forced MRT)
    // Smagorinsky: tau = tau + tau_sgs with tau_sgs from the non-equilibrium stress
    int les;
    double les_c;           // 18 Cs^2
    const float* c_node;    // learned closure: per-cell constant c (C = 18 c), or nullptr
    double conv_u[6];       // convective outflow: convection speed per face
    // FP16 / BF16 stochastic rounding: two step seeds of the level in device memory (the even
    // step reads [0] and its first thread writes [1] = [0] + 1, the odd step the other way round,
    // so no launch reads a word another thread of it writes); nullptr: round to nearest
    uint32_t* sr_seed;
};

// ---------------------------------------------------------------- stochastic rounding
// Random bits for stochastic rounding: a counter-based stream per thread, seeded by the step
// seed and the thread's node (or node pair, or lane) index through the "lowbias32" integer hash
// (C. Wellons, 2018, public domain), advanced by a 32-bit linear congruential step (the
// Numerical Recipes constants) whose output is folded (x ^ x >> 16) so that its low bits are
// usable.  Deterministic: the same calls give the same bits.
struct SrBits {
    uint32_t h;
    __device__ __forceinline__ static uint32_t mix(uint32_t x) {
        x ^= x >> 16;
        x *= 0x7feb352du;
        x ^= x >> 15;
        x *= 0x846ca68bu;
        x ^= x >> 16;
        return x;
    }
    __device__ __forceinline__ SrBits(uint32_t seed, uint32_t stream) : h(mix(mix(seed) ^ stream)) {}
    __device__ __forceinline__ uint32_t next() {
        h = h * 1664525u + 1013904223u;
        return h ^ (h >> 16);
    }
};

// The level's step seed for this layout phase, and its advance by the launch's first thread.
__device__ __forceinline__ uint32_t sr_seed(const StepParams& p, bool odd) {
    return p.sr_seed ? __ldcg(p.sr_seed + (odd ? 1 : 0)) : 0u;
}
__device__ __forceinline__ void sr_advance(const StepParams& p, bool odd, uint32_t seed, bool leader) {
    if (p.sr_seed && leader) p.sr_seed[odd ? 0 : 1] = seed + 1u;
}

// FP32 -> FP16 / BF16 pairs with the sm_100 stochastic-rounding conversion (cvt.rs, random bits
// from rbits); the first operand lands in the upper half, as with cvt.rn
__device__ __forceinline__ uint32_t cvt_rs_f16x2(float hi, float lo, uint32_t rbits) {
    uint32_t d;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    return d;
}
__device__ __forceinline__ uint32_t cvt_rs_bf16x2(float hi, float lo, uint32_t rbits) {
    uint32_t d;
    asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    return d;
}

// Per-node extras handed to the collision.
struct NodeForce {
    double F[3];
};

// ---------------------------------------------------------------- storage
template <class S> struct Storage;
template <> struct Storage<double> {
    using T = double;
    static constexpr bool kDeviation = false;
    static constexpr bool kScaled = false;
    ZL_HD static T load_raw(const double* p) { return *p; }
    ZL_HD static void store_raw(double* p, T v) { *p = v; }
    ZL_HD static void store_raw_sr(double* p, T v, uint32_t) { *p = v; }
    ZL_HD static T load(const double* p, const StepParams&) { return *p; }
    ZL_HD static void store(double* p, T v, const StepParams&) { *p = v; }
};
template <> struct Storage<float> {
    using T = float;
    static constexpr bool kDeviation = true;
    static constexpr bool kScaled = false;
    __device__ __forceinline__ static T load_raw(const float* p) { return __ldg(p); }
    __device__ __forceinline__ static void store_raw(float* p, T v) { *p = v; }
    __device__ __forceinline__ static void store_raw_sr(float* p, T v, uint32_t) { *p = v; }
    __device__ __forceinline__ static T load(const float* p, const StepParams&) { return __ldg(p); }
    __device__ __forceinline__ static void store(float* p, T v, const StepParams&) { *p = v; }
};
// Reduced storage keeps (f - w) * scale.  The fused step kernel works directly in these
// scaled units (the collision is linear in the deviations apart from the equilibrium, which
// un-scales density and momentum once), so only the exchange and boundary kernels apply the
// scale per population.
template <> struct Storage<__half> {
    using T = float;
    static constexpr bool kDeviation = true;
    static constexpr bool kScaled = true;
    __device__ __forceinline__ static T load_raw(const __half* p) { return __half2float(__ldg(p)); }
    __device__ __forceinline__ static void store_raw(__half* p, T v) { *p = __float2half_rn(v); }
    __device__ __forceinline__ static void store_raw_sr(__half* p, T v, uint32_t rbits) {
        const unsigned short h = (unsigned short)(cvt_rs_f16x2(0.f, v, rbits) & 0xffffu);
        *reinterpret_cast<unsigned short*>(p) = h;
    }
    __device__ __forceinline__ static T load(const __half* p, const StepParams& sp) {
        return load_raw(p) * sp.inv_scale;
    }
    __device__ __forceinline__ static void store(__half* p, T v, const StepParams& sp) { store_raw(p, v * sp.scale); }
};
template <> struct Storage<__nv_bfloat16> {
    using T = float;
    static constexpr bool kDeviation = true;
    static constexpr bool kScaled = true;
    __device__ __forceinline__ static T load_raw(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }
    __device__ __forceinline__ static void store_raw(__nv_bfloat16* p, T v) { *p = __float2bfloat16_rn(v); }
    __device__ __forceinline__ static void store_raw_sr(__nv_bfloat16* p, T v, uint32_t rbits) {
        const unsigned short h = (unsigned short)(cvt_rs_bf16x2(0.f, v, rbits) & 0xffffu);
        *reinterpret_cast<unsigned short*>(p) = h;
    }
    __device__ __forceinline__ static T load(const __nv_bfloat16* p, const StepParams& sp) {
        return load_raw(p) * sp.inv_scale;
    }
    __device__ __forceinline__ static void store(__nv_bfloat16* p, T v, const StepParams& sp) {
        store_raw(p, v * sp.scale);
    }
};

// ---------------------------------------------------------------- collision
// Exact FP64 path: reference arithmetic order (lbm_solver_interface.cpp:374-435, :477-532,
// collision_model/lbm_collision_model_srt.cpp:20-25, lbm_collision_model_mrt.cpp:114-125).
// Compiled with -fmad=false so that no product is fused into an FMA.  Terms the
// reference multiplies by a zero lattice component add +-0 and are skipped: that
// leaves every sum bit-identical.
template <class L>
__device__ __forceinline__ void macro_exact(const double* f, double& rho, double& ux, double& uy, double& uz,
                                            const double* F = nullptr, double dt = 0.) {
    using Tb = Tables<L>;
    rho = f[0];
    ux = 0.;
    uy = 0.;
    uz = 0.;
#pragma unroll
    for (int q = 1; q < L::kQ; ++q) {
        rho = rho + f[q];
        if (Tb::cx(q) == 1) ux = ux + f[q];
        if (Tb::cx(q) == -1) ux = ux - f[q];
        if (Tb::cy(q) == 1) uy = uy + f[q];
        if (Tb::cy(q) == -1) uy = uy - f[q];
        if (L::kDims == 3) {
            if (Tb::cz(q) == 1) uz = uz + f[q];
            if (Tb::cz(q) == -1) uz = uz - f[q];
        }
    }
    if (F) {
        // CalMacroForce{2D,3D}Incompressible (lbm_solver_interface.cpp:556-561, :586-592)
        ux = ux + 0.5 * F[0] * dt;
        uy = uy + 0.5 * F[1] * dt;
        if (L::kDims == 3) uz = uz + 0.5 * F[2] * dt;
    }
    ux = ux / rho;
    uy = uy / rho;
    if (L::kDims == 3) uz = uz / rho;
}

template <class L>
__device__ __forceinline__ void feq_exact(double rho, double ux, double uy, double uz, double* feq) {
    using Tb = Tables<L>;
    const double uv_sq = L::kDims == 3 ? (ux * ux + uy * uy) + uz * uz : ux * ux + uy * uy;
#pragma unroll
    for (int q = 0; q < L::kQ; ++q) {
        // c.u over the non-zero components in x, y, z order
        double cu = 0.;
        bool first = true;
        if (Tb::cx(q) != 0) {
            cu = Tb::cx(q) == 1 ? ux : -ux;
            first = false;
        }
        if (Tb::cy(q) != 0) {
            const double t = Tb::cy(q) == 1 ? uy : -uy;
            cu = first ? t : cu + t;
            first = false;
        }
        if (L::kDims == 3 && Tb::cz(q) != 0) {
            const double t = Tb::cz(q) == 1 ? uz : -uz;
            cu = first ? t : cu + t;
            first = false;
        }
        const double wr = Tb::w(q) * rho;
        feq[q] = wr * (((1. + 3. * cu) + (4.5 * cu) * cu) - 1.5 * uv_sq);
    }
}

// Smagorinsky subgrid relaxation increment in the reference's arithmetic
// (les_models/lbm_les_smagorinsky.cpp:22-94); u is the node velocity used by the collision.
template <class L>
__device__ __forceinline__ double smag_tau_sgs_exact(const double* f, const double* feq, double tau0, double c,
                                                     bool forced, const double* F, double dt, double ux, double uy,
                                                     double uz) {
    using Tb = Tables<L>;
    double pxx = 0., pxy = 0., pyy = 0., pzz = 0., pxz = 0., pyz = 0.;
#pragma unroll
    for (int q = 1; q < L::kQ; ++q) {
        const double cx = Tb::cx(q), cy = Tb::cy(q), cz = Tb::cz(q);
        const double d = f[q] - feq[q];
        pxx += cx * cx * d;
        pxy += cx * cy * d;
        pyy += cy * cy * d;
        if (L::kDims == 3) {
            pzz += cz * cz * d;
            pxz += cx * cz * d;
            pyz += cy * cz * d;
        }
    }
    if (forced) {
        pxx += dt * F[0] * ux;
        pyy += dt * F[1] * uy;
        pxy += 0.5 * dt * (F[0] * ux + F[1] * uy);
        if (L::kDims == 3) {
            pzz += dt * F[2] * uz;
            pxz += 0.5 * dt * (F[0] * ux + F[2] * uz);
            pyz += 0.5 * dt * (F[1] * uy + F[2] * uz);
        }
    }
    const double pi2 = pxx * pxx + pyy * pyy + pzz * pzz + 2. * (pxy * pxy + pxz * pxz + pyz * pyz);
    return 0.5 * (sqrt(tau0 * tau0 + c * sqrt(2. * pi2)) - tau0);
}

// Element (q, s) of M^-1 S M (d_matrix: M^-1 (I - S/2) M) for relaxation 1/tau, summed over the
// moments in the reference's order (collision_model/lbm_collision_model_mrt.cpp:63-107).
template <class L>
__device__ __forceinline__ double mrt_element_exact(int q, int s, double relax, bool d_matrix) {
    using Tb = Tables<L>;
    double acc = 0.;
#pragma unroll
    for (int k = 0; k < L::kQ; ++k) {
        double sk = Tb::s(k) < 0. ? relax : Tb::s(k);
        if (d_matrix) sk = 1. - 0.5 * sk;
        const double im = (double)Tb::M(k, q) / (double)row_norm2<L>(k);
        acc = acc + im * (sk * (double)Tb::M(k, s));
    }
    return acc;
}

template <class L, bool Les>
__device__ __forceinline__ void collide_exact(const double* f, double* out, const StepParams& p, int coll,
                                              double* mac, const NodeForce* nf) {
    using Tb = Tables<L>;
    constexpr int Q = L::kQ;
    double rho, ux, uy, uz;
    if (nf) {
        // CalMacroForce*Compressible (lbm_solver_interface.cpp:541-592): u += 0.5 F dt before / rho
        rho = f[0];
        ux = 0.;
        uy = 0.;
        uz = 0.;
#pragma unroll
        for (int q = 1; q < Q; ++q) {
            rho = rho + f[q];
            if (Tb::cx(q) == 1) ux = ux + f[q];
            if (Tb::cx(q) == -1) ux = ux - f[q];
            if (Tb::cy(q) == 1) uy = uy + f[q];
            if (Tb::cy(q) == -1) uy = uy - f[q];
            if (L::kDims == 3) {
                if (Tb::cz(q) == 1) uz = uz + f[q];
                if (Tb::cz(q) == -1) uz = uz - f[q];
            }
        }
        ux = ux + 0.5 * nf->F[0] * p.dt;
        uy = uy + 0.5 * nf->F[1] * p.dt;
        if (L::kDims == 3) uz = uz + 0.5 * nf->F[2] * p.dt;
        ux = ux / rho;
        uy = uy / rho;
        if (L::kDims == 3) uz = uz / rho;
    } else {
        macro_exact<L>(f, rho, ux, uy, uz);
    }
    mac[0] = rho;
    mac[1] = ux;
    mac[2] = uy;
    mac[3] = uz;
    double feq[Q];
    feq_exact<L>(rho, ux, uy, uz, feq);
    double fterm[Q];
    if (nf) {
        // CalForcingTerming2D/3D (lbm_solver_interface.cpp:443-470)
        const double* F = nf->F;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const double cx = Tb::cx(q), cy = Tb::cy(q), cz = Tb::cz(q);
            if (L::kDims == 2) {
                fterm[q] = Tb::w(q) * (3. * ((cx - ux) * F[0] + (cy - uy) * F[1])
                                       + 9. * (ux * cx + uy * cy) * (cx * F[0] + cy * F[1]));
            } else {
                fterm[q] = Tb::w(q) * (3. * ((cx - ux) * F[0] + (cy - uy) * F[1] + (cz - uz) * F[2])
                                       + 9. * (ux * cx + uy * cy + uz * cz) * (cx * F[0] + cy * F[1] + cz * F[2]));
            }
        }
    }
    double tau = p.tau;
    if (Les) tau = p.tau + smag_tau_sgs_exact<L>(f, feq, p.tau, p.les_c, nf != nullptr, nf ? nf->F : nullptr,
                                                   p.dt, ux, uy, uz);
    if (coll == kSrt) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            if (nf)
                out[q] = f[q] - (f[q] - feq[q]) / tau + (1. - 0.5 / tau) * fterm[q] * p.dt;
            else
                out[q] = f[q] - (f[q] - feq[q]) / tau;
        }
    } else {
        double d[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) d[q] = f[q] - feq[q];
        if (!Les) {
            const double* A = p.mrt64;
            const double* B = p.mrt64_d;
#pragma unroll 1
            for (int q = 0; q < Q; ++q) {
                double acc = 0.;
                if (nf) {
#pragma unroll
                    for (int s = 0; s < Q; ++s)
                        acc += __ldg(A + q * Q + s) * d[s] - __ldg(B + q * Q + s) * fterm[s] * p.dt;
                } else {
#pragma unroll
                    for (int s = 0; s < Q; ++s) acc = acc + __ldg(A + q * Q + s) * d[s];
                }
                out[q] = f[q] - acc;
            }
        } else {
            // the relaxation time differs per node: build M^-1 S M on the fly
            const double relax = 1. / tau;
#pragma unroll 1
            for (int q = 0; q < Q; ++q) {
                double acc = 0.;
#pragma unroll 1
                for (int s = 0; s < Q; ++s) {
                    const double a = mrt_element_exact<L>(q, s, relax, false);
                    if (nf) {
                        const double b = mrt_element_exact<L>(q, s, relax, true);
                        acc += a * d[s] - b * fterm[s] * p.dt;
                    } else {
                        acc = acc + a * d[s];
                    }
                }
                out[q] = f[q] - acc;
            }
        }
    }
}

// Fast path on deviations d_q = f_q - w_q, FP32 arithmetic.
//
// MRT as f* = f - S_nu neq - sum_k lambda_k m_k M_k^T over the moments whose rate differs
// from the shear rate S_nu = 1/tau (the basis is orthogonal, so the shear moments fold into
// the first term); lambda_k = (s_k - 1/tau) / |M_k|^2 and m_k = M_k . neq.  The conserved
// moments of neq vanish and are skipped.
// c_q . u with the zero components left out (a product with 0.f is not folded away under IEEE rules)
template <class L>
__device__ __forceinline__ float signed_dot(int q, float ux, float uy, float uz) {
    using Tb = Tables<L>;
    float cu = 0.f;
    bool first = true;
    if (Tb::cx(q)) { cu = Tb::cx(q) > 0 ? ux : -ux; first = false; }
    if (Tb::cy(q)) { cu = first ? (Tb::cy(q) > 0 ? uy : -uy) : (Tb::cy(q) > 0 ? cu + uy : cu - uy); first = false; }
    if (L::kDims == 3 && Tb::cz(q)) { cu = first ? (Tb::cz(q) > 0 ? uz : -uz) : (Tb::cz(q) > 0 ? cu + uz : cu - uz); }
    return cu;
}

template <class L>
__device__ __forceinline__ void feq_neq_dev(const float* d, float* neq, float scale, float inv_scale, float* mac,
                                            const float* F = nullptr, float dt = 0.f) {
    // d are deviations times `scale`; neq is returned in the same units; F (unscaled) shifts the
    // velocity by F dt / 2 (Guo forcing)
    using Tb = Tables<L>;
    constexpr int Q = L::kQ;
    float drho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        drho += d[q];
        if (Tb::cx(q)) jx += Tb::cx(q) == 1 ? d[q] : -d[q];
        if (Tb::cy(q)) jy += Tb::cy(q) == 1 ? d[q] : -d[q];
        if (L::kDims == 3 && Tb::cz(q)) jz += Tb::cz(q) == 1 ? d[q] : -d[q];
    }
    const float rho = fmaf(drho, inv_scale, 1.f);
    const float k = inv_scale / rho;
    float ux = jx * k, uy = jy * k, uz = jz * k;
    if (F) {
        const float h = 0.5f * dt / rho;
        ux = fmaf(h, F[0], ux);
        uy = fmaf(h, F[1], uy);
        uz = fmaf(h, F[2], uz);
    }
    mac[0] = rho;
    mac[1] = ux;
    mac[2] = uy;
    mac[3] = uz;
    const float usq15 = 1.5f * (ux * ux + uy * uy + uz * uz);
    const float srho = scale * rho;
    // even part shared by opposite directions, odd part 3 w rho (c.u)
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int opp = Tb::opp(q);
        if (opp < q) continue;
        const float cu = signed_dot<L>(q, ux, uy, uz);
        const float w = (float)Tb::w(q);
        const float even = w * fmaf(srho, fmaf(4.5f * cu, cu, -usq15), drho);
        if (q == 0) {
            neq[0] = d[0] - even;
        } else {
            const float odd = (3.f * w) * srho * cu;
            neq[q] = d[q] - (even + odd);
            neq[opp] = d[opp] - (even - odd);
        }
    }
}

__device__ __forceinline__ void mrt_d3q19_dev(const float* d, const float* n, float* out, float omega,
                                              const float* lam) {
    // pair sums / differences over opposite directions
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
    const float m1 = -30.f * n[0] - 11.f * Sa + 8.f * Sd;
    const float m2 = 12.f * n[0] - 4.f * Sa + Sd;
    const float m10 = -4.f * S1 + 2.f * (S2 + S3) + Sxy + Sxz - 2.f * Syz;
    const float m12 = -2.f * S2 + 2.f * S3 + Sxy - Sxz;
    const float X1 = D4 - D5, X2 = D6 - D7;
    const float Y1 = D4 + D5, Y2 = D8 - D9;
    const float Z1 = D6 + D7, Z2 = D8 + D9;
    const float m4 = -4.f * D1 + X1 + X2, m16 = X1 - X2;
    const float m6 = -4.f * D2 + Y1 + Y2, m17 = -Y1 + Y2;
    const float m8 = -4.f * D3 + Z1 + Z2, m18 = Z1 - Z2;
    // lambda_k = (s_k - omega) / |M_k|^2
    const float a1 = lam[1] * m1, a2 = lam[2] * m2;
    const float a4 = lam[4] * m4, a6 = lam[6] * m6, a8 = lam[8] * m8;
    const float a10 = lam[10] * m10, a12 = lam[12] * m12;
    const float a16 = lam[16] * m16, a17 = lam[17] * m17, a18 = lam[18] * m18;
    const float e_ax = -11.f * a1 - 4.f * a2;
    const float e_dg = 8.f * a1 + a2;
    float c[19];
    c[0] = -30.f * a1 + 12.f * a2;
    {
        const float E = e_ax - 4.f * a10, O = -4.f * a4;
        c[1] = E + O; c[2] = E - O;
    }
    {
        const float E = e_ax + 2.f * a10 - 2.f * a12, O = -4.f * a6;
        c[3] = E + O; c[4] = E - O;
    }
    {
        const float E = e_ax + 2.f * a10 + 2.f * a12, O = -4.f * a8;
        c[5] = E + O; c[6] = E - O;
    }
    const float e_xy = e_dg + a10 + a12, e_xz = e_dg + a10 - a12, e_yz = e_dg - 2.f * a10;
    {
        const float O = a4 + a6 + a16 - a17;   // q = 7 (+1,+1,0), opposite 10
        c[7] = e_xy + O; c[10] = e_xy - O;
    }
    {
        const float O = -a4 + a6 - a16 - a17;  // q = 8 (-1,+1,0), opposite 9
        c[8] = e_xy + O; c[9] = e_xy - O;
    }
    {
        const float O = a4 + a8 - a16 + a18;   // q = 11 (+1,0,+1), opposite 14
        c[11] = e_xz + O; c[14] = e_xz - O;
    }
    {
        const float O = -a4 + a8 + a16 + a18;  // q = 12 (-1,0,+1), opposite 13
        c[12] = e_xz + O; c[13] = e_xz - O;
    }
    {
        const float O = a6 + a8 + a17 - a18;   // q = 15 (0,+1,+1), opposite 18
        c[15] = e_yz + O; c[18] = e_yz - O;
    }
    {
        const float O = -a6 + a8 - a17 - a18;  // q = 16 (0,-1,+1), opposite 17
        c[16] = e_yz + O; c[17] = e_yz - O;
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) out[q] = fmaf(-omega, n[q], d[q]) - c[q];
}

// D3Q19 SRT, optionally with Smagorinsky and with a Guo body force F (Forced), in one pass over
// the deviations d (scaled units): the pair sums / differences of opposite directions give the
// density, momentum and second moments; the non-equilibrium stress of the reference's second-
// order equilibrium (lbm_solver_interface.cpp:374-435) is then
// Pi_ab = sum_q c_a c_b d_q - drho / 3 delta_ab - G u_a u_b (G = scale rho), its diagonal sums
// S1 + Sxy + Sxz (x), ... and its off-diagonal S4 - S5 (xy), S6 - S7 (xz), S8 - S9 (yz).
// Smagorinsky: tau = tau0 + (sqrt(tau0^2 + C sqrt(2 Pi:Pi)) - tau0) / 2
// (lbm_les_smagorinsky.cpp:22-94 with the increment added to tau0).  The update
// f*_q = (1 - omega) d_q + omega feq_q (+ (1 - omega / 2) dt Fq_q) is formed per opposite pair
// from its sum and difference: feq_q = w (B + 4.5 G (c.u)^2) + 3 w (c.j), B = drho - 1.5 G u^2.
// With a force (CalMacroForce*, CalForcingTerming3D: lbm_solver_interface.cpp:443-470, 541-592)
// the velocity is shifted by F dt / (2 rho), j is G u, the stress gains dt (F_a u_b + F_b u_a) / 2,
// and Fq_q = w [3 (c - u).F + 9 (c.u)(c.F)] splits into an even part w (9 (c.u)(c.F) - 3 u.F) and
// an odd part 3 w (c.F) per pair: the same update as the general forced path (feq_neq_dev and the
// per-direction Guo term), in another rounding order.
template <bool Forced>
__device__ __forceinline__ void srt_d3q19_fused_t(const float* d, float* out, const StepParams& p, float* mac,
                                                  bool les, float les_c, const float* F) {
    const float S1 = d[1] + d[2], D1 = d[1] - d[2];
    const float S2 = d[3] + d[4], D2 = d[3] - d[4];
    const float S3 = d[5] + d[6], D3 = d[5] - d[6];
    const float S4 = d[7] + d[10], D4 = d[7] - d[10];
    const float S5 = d[8] + d[9], D5 = d[8] - d[9];
    const float S6 = d[11] + d[14], D6 = d[11] - d[14];
    const float S7 = d[12] + d[13], D7 = d[12] - d[13];
    const float S8 = d[15] + d[18], D8 = d[15] - d[18];
    const float S9 = d[16] + d[17], D9 = d[16] - d[17];
    const float Sxy = S4 + S5, Sxz = S6 + S7, Syz = S8 + S9;
    const float drho = ((d[0] + S1) + (S2 + S3)) + ((Sxy + Sxz) + Syz);
    float jx = D1 + (D4 - D5) + (D6 - D7);
    float jy = D2 + (D4 + D5) + (D8 - D9);
    float jz = D3 + (D6 + D7) + (D8 + D9);
    const float rho = fmaf(drho, p.inv_scale, 1.f);
    float ux, uy, uz;
    if constexpr (Forced) {
        const float k = p.inv_scale / rho, h = 0.5f * (float)p.dt / rho;
        ux = fmaf(h, F[0], jx * k);
        uy = fmaf(h, F[1], jy * k);
        uz = fmaf(h, F[2], jz * k);
    } else {
        const float k = __fdividef(p.inv_scale, rho);  // fast reciprocal, two ulps (rho is close to 1)
        ux = jx * k;
        uy = jy * k;
        uz = jz * k;
    }
    mac[0] = rho;
    mac[1] = ux;
    mac[2] = uy;
    mac[3] = uz;
    const float ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
    const float G = p.scale * rho;
    if constexpr (Forced) {
        // the momentum of the shifted equilibrium
        jx = G * ux;
        jy = G * uy;
        jz = G * uz;
    }
    float omega = p.omega32;
    if (les) {
        const float t = drho * (1.f / 3.f);
        float pxx = fmaf(-G, ux2, (S1 + Sxy + Sxz) - t);
        float pyy = fmaf(-G, uy2, (S2 + Sxy + Syz) - t);
        float pzz = fmaf(-G, uz2, (S3 + Sxz + Syz) - t);
        float pxy = fmaf(-G, ux * uy, S4 - S5);
        float pxz = fmaf(-G, ux * uz, S6 - S7);
        float pyz = fmaf(-G, uy * uz, S8 - S9);
        if constexpr (Forced) {
            const float ds = (float)p.dt * p.scale;
            const float fx = ds * F[0] * ux, fy = ds * F[1] * uy, fz = ds * F[2] * uz;
            pxx += fx;
            pyy += fy;
            pzz += fz;
            pxy += 0.5f * (fx + fy);
            pxz += 0.5f * (fx + fz);
            pyz += 0.5f * (fy + fz);
        }
        const float is2 = p.inv_scale * p.inv_scale;
        const float pi2 = is2 * (pxx * pxx + pyy * pyy + pzz * pzz + 2.f * (pxy * pxy + pxz * pxz + pyz * pyz));
        const float tau0 = (float)p.tau;
        const float tau = tau0 + 0.5f * (sqrtf(tau0 * tau0 + les_c * sqrtf(2.f * pi2)) - tau0);
        omega = 1.f / tau;
    }
    const float B = fmaf(-1.5f * G, ux2 + uy2 + uz2, drho);
    const float h = 0.5f * (1.f - omega);
    const float ow0 = omega * (1.f / 3.f), ow1 = omega * (1.f / 18.f), ow2 = omega * (1.f / 36.f);
    const float K1 = 4.5f * ow1 * G, L1 = ow1 * B, o1 = 3.f * ow1;
    const float K2 = 4.5f * ow2 * G, L2 = ow2 * B, o2 = 3.f * ow2;
    // Guo term parts, scaled: gF_w = (1 - omega/2) dt scale w
    float g1 = 0.f, g2 = 0.f, uF3 = 0.f;
    if constexpr (Forced) {
        const float g = (1.f - 0.5f * omega) * (float)p.dt * p.scale;
        g1 = g * (1.f / 18.f);
        g2 = g * (1.f / 36.f);
        uF3 = 3.f * (ux * F[0] + uy * F[1] + uz * F[2]);
        out[0] = fmaf(1.f - omega, d[0], fmaf(ow0, B, -(g * (1.f / 3.f)) * uF3));
    } else {
        out[0] = fmaf(1.f - omega, d[0], ow0 * B);
    }
    auto pair = [&](int q, int o, float S, float D, float even, float odd) {
        const float e = fmaf(h, S, even), od = fmaf(h, D, odd);
        out[q] = e + od;
        out[o] = e - od;
    };
    // (even, odd) Guo parts of a pair with c.u = cu, c.F = cF and weight factor gw
    auto force = [&](float gw, float cu, float cF, float& even, float& odd) {
        if constexpr (Forced) {
            even = fmaf(gw, fmaf(9.f * cu, cF, -uF3), even);
            odd = fmaf(gw * 3.f, cF, odd);
        }
    };
    {
        float e1 = fmaf(K1, ux2, L1), od1 = o1 * jx, e2 = fmaf(K1, uy2, L1), od2 = o1 * jy;
        float e3 = fmaf(K1, uz2, L1), od3 = o1 * jz;
        if constexpr (Forced) {
            force(g1, ux, F[0], e1, od1);
            force(g1, uy, F[1], e2, od2);
            force(g1, uz, F[2], e3, od3);
        }
        pair(1, 2, S1, D1, e1, od1);
        pair(3, 4, S2, D2, e2, od2);
        pair(5, 6, S3, D3, e3, od3);
    }
    {
        const float a = ux + uy, b = uy - ux;
        float ea = fmaf(K2, a * a, L2), oa = o2 * (jx + jy), eb = fmaf(K2, b * b, L2), ob = o2 * (jy - jx);
        if constexpr (Forced) {
            force(g2, a, F[0] + F[1], ea, oa);
            force(g2, b, F[1] - F[0], eb, ob);
        }
        pair(7, 10, S4, D4, ea, oa);
        pair(8, 9, S5, D5, eb, ob);
    }
    {
        const float a = ux + uz, b = uz - ux;
        float ea = fmaf(K2, a * a, L2), oa = o2 * (jx + jz), eb = fmaf(K2, b * b, L2), ob = o2 * (jz - jx);
        if constexpr (Forced) {
            force(g2, a, F[0] + F[2], ea, oa);
            force(g2, b, F[2] - F[0], eb, ob);
        }
        pair(11, 14, S6, D6, ea, oa);
        pair(12, 13, S7, D7, eb, ob);
    }
    {
        const float a = uy + uz, b = uz - uy;
        float ea = fmaf(K2, a * a, L2), oa = o2 * (jy + jz), eb = fmaf(K2, b * b, L2), ob = o2 * (jz - jy);
        if constexpr (Forced) {
            force(g2, a, F[1] + F[2], ea, oa);
            force(g2, b, F[2] - F[1], eb, ob);
        }
        pair(15, 18, S8, D8, ea, oa);
        pair(16, 17, S9, D9, eb, ob);
    }
}

__device__ __forceinline__ void srt_d3q19_fused(const float* d, float* out, const StepParams& p, float* mac,
                                                bool les, float les_c) {
    srt_d3q19_fused_t<false>(d, out, p, mac, les, les_c, nullptr);
}

// D3Q19 MRT without forcing or LES, in one pass over the deviations d (scaled units).
//
// The same update as feq_neq_dev + mrt_d3q19_dev, f* = f - omega neq - sum_k lambda_k m_k M_k,
// rearranged so that no per-direction neq is formed:
//   * the relaxed moments of neq are the moments of d minus their equilibrium values, which are
//     closed forms in (rho, j) for the second-order equilibrium of the reference
//     (lbm_solver_interface.cpp:374-435): with drho = scale (rho - 1), G = scale rho,
//     m1 = 19 (Sd - d0 - G u^2), m2 = 9 d0 - 7 Sa - 2 Sd + 5.5 G u^2,
//     m4 = -(10/3) D1 + (5/3)(X1 + X2) (likewise m6, m8: -2/3 j folded in),
//     m10 = M10.d + G (3 ux^2 - u^2) / 2, m12 = M12.d + G (uy^2 - uz^2) / 2, m16..18 = M.d;
//   * f*_q = (1 - omega) d_q + omega feq_q - c_q, with d_q, feq_q and c_q split into the parts
//     even and odd under q -> opp(q), so each opposite pair is formed from its sum and difference
//     (the populations themselves are not needed past the pair sums).
// The odd part of feq uses the momentum sums j directly (3 w G (c.u) = 3 w (c.j)).
__device__ __forceinline__ void mrt_d3q19_fused(const float* d, float* out, const StepParams& p, float* mac) {
    const float omega = p.omega32;
    const float* lam = p.mrt_coef;
    const float S1 = d[1] + d[2], D1 = d[1] - d[2];
    const float S2 = d[3] + d[4], D2 = d[3] - d[4];
    const float S3 = d[5] + d[6], D3 = d[5] - d[6];
    const float S4 = d[7] + d[10], D4 = d[7] - d[10];
    const float S5 = d[8] + d[9], D5 = d[8] - d[9];
    const float S6 = d[11] + d[14], D6 = d[11] - d[14];
    const float S7 = d[12] + d[13], D7 = d[12] - d[13];
    const float S8 = d[15] + d[18], D8 = d[15] - d[18];
    const float S9 = d[16] + d[17], D9 = d[16] - d[17];
    const float S23 = S2 + S3;
    const float Sa = S1 + S23;
    const float Sxy = S4 + S5, Sxz = S6 + S7, Syz = S8 + S9;
    const float Sd = (Sxy + Sxz) + Syz;
    const float drho = (d[0] + Sa) + Sd;
    const float X1 = D4 - D5, X2 = D6 - D7;
    const float Y1 = D4 + D5, Y2 = D8 - D9;
    const float Z1 = D6 + D7, Z2 = D8 + D9;
    const float X12 = X1 + X2, Y12 = Y1 + Y2, Z12 = Z1 + Z2;
    const float jx = D1 + X12, jy = D2 + Y12, jz = D3 + Z12;
    const float rho = fmaf(drho, p.inv_scale, 1.f);
    const float k = __fdividef(p.inv_scale, rho);  // fast reciprocal, two ulps (rho is close to 1)
    const float ux = jx * k, uy = jy * k, uz = jz * k;
    mac[0] = rho;
    mac[1] = ux;
    mac[2] = uy;
    mac[3] = uz;
    const float ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
    const float usq = ux2 + uy2 + uz2;
    const float G = p.scale * rho;
    const float Gu = G * usq;
    // relaxed moments of neq, times lambda_k = (s_k - omega) / |M_k|^2
    const float a1 = (19.f * lam[1]) * ((Sd - d[0]) - Gu);
    const float a2 = lam[2] * fmaf(5.5f, Gu, fmaf(9.f, d[0], fmaf(-7.f, Sa, -2.f * Sd)));
    const float a4 = lam[4] * fmaf(-10.f / 3.f, D1, (5.f / 3.f) * X12);
    const float a6 = lam[6] * fmaf(-10.f / 3.f, D2, (5.f / 3.f) * Y12);
    const float a8 = lam[8] * fmaf(-10.f / 3.f, D3, (5.f / 3.f) * Z12);
    const float hG = 0.5f * G;
    const float a10 = lam[10] * fmaf(hG, fmaf(3.f, ux2, -usq), fmaf(-4.f, S1, fmaf(2.f, S23, (Sxy + Sxz) - 2.f * Syz)));
    const float a12 = lam[12] * fmaf(hG, uy2 - uz2, fmaf(2.f, S3 - S2, Sxy - Sxz));
    const float a16 = lam[16] * (X1 - X2), a17 = lam[17] * (Y2 - Y1), a18 = lam[18] * (Z1 - Z2);
    // even parts of the correction per direction class, odd parts per pair
    const float e_ax = fmaf(-11.f, a1, -4.f * a2);
    const float e_dg = fmaf(8.f, a1, a2);
    const float c0 = fmaf(-30.f, a1, 12.f * a2);
    const float cx = fmaf(-4.f, a10, e_ax);
    const float cy = e_ax + 2.f * (a10 - a12);
    const float cz = e_ax + 2.f * (a10 + a12);
    const float c_xy = e_dg + (a10 + a12), c_xz = e_dg + (a10 - a12), c_yz = fmaf(-2.f, a10, e_dg);
    const float u1 = a4 + a16, u2 = a6 - a17;   // q7: u1 + u2, q8: u2 - u1
    const float v1 = a4 - a16, v2 = a8 + a18;   // q11: v1 + v2, q12: v2 - v1
    const float t1 = a6 + a17, t2 = a8 - a18;   // q15: t1 + t2, q16: t2 - t1
    // omega feq: w (B + 4.5 G (c.u)^2) even, 3 w (c.j) odd, B = drho - 1.5 G u^2
    const float B = fmaf(-1.5f, Gu, drho);
    const float ow0 = omega * (1.f / 3.f), ow1 = omega * (1.f / 18.f), ow2 = omega * (1.f / 36.f);
    const float K1 = ow1 * (4.5f * G), L1 = ow1 * B;
    const float K2 = ow2 * (4.5f * G), L2 = ow2 * B, K2x2 = K2 + K2;
    const float o1 = ow1 * 3.f, o2 = ow2 * 3.f;
    // (1 - omega) d_q of a pair from its sum and difference: d_q = (S + D) / 2, d_opp = (S - D) / 2
    const float h = 0.5f * (1.f - omega);
    out[0] = fmaf(1.f - omega, d[0], fmaf(ow0, B, -c0));
    auto pair = [&](int q, int o, float S, float D, float A, float Bo) {
        const float e = fmaf(h, S, A), od = fmaf(h, D, Bo);
        out[q] = e + od;
        out[o] = e - od;
    };
    pair(1, 2, S1, D1, fmaf(K1, ux2, L1) - cx, fmaf(o1, jx, 4.f * a4));
    pair(3, 4, S2, D2, fmaf(K1, uy2, L1) - cy, fmaf(o1, jy, 4.f * a6));
    pair(5, 6, S3, D3, fmaf(K1, uz2, L1) - cz, fmaf(o1, jz, 4.f * a8));
    {
        // xy plane: q7 (+1,+1,0) / q10, q8 (-1,+1,0) / q9
        const float P = fmaf(K2, ux2 + uy2, L2) - c_xy, Q = K2x2 * (ux * uy);
        pair(7, 10, S4, D4, P + Q, fmaf(o2, jx + jy, -(u1 + u2)));
        pair(8, 9, S5, D5, P - Q, fmaf(o2, jy - jx, -(u2 - u1)));
    }
    {
        // xz plane: q11 (+1,0,+1) / q14, q12 (-1,0,+1) / q13
        const float P = fmaf(K2, ux2 + uz2, L2) - c_xz, Q = K2x2 * (ux * uz);
        pair(11, 14, S6, D6, P + Q, fmaf(o2, jx + jz, -(v1 + v2)));
        pair(12, 13, S7, D7, P - Q, fmaf(o2, jz - jx, -(v2 - v1)));
    }
    {
        // yz plane: q15 (0,+1,+1) / q18, q16 (0,-1,+1) / q17
        const float P = fmaf(K2, uy2 + uz2, L2) - c_yz, Q = K2x2 * (uy * uz);
        pair(15, 18, S8, D8, P + Q, fmaf(o2, jy + jz, -(t1 + t2)));
        pair(16, 17, S9, D9, P - Q, fmaf(o2, jz - jy, -(t2 - t1)));
    }
}

// out_q = sum_k coef_k (M_k . x) M_kq over the moments flagged in `use` (compile-time folded basis).
template <class L, class Use>
__device__ __forceinline__ void moment_apply(const float* x, const float* coef, float* out, Use use) {
    using Tb = Tables<L>;
    constexpr int Q = L::kQ;
    float a[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        float acc = 0.f;
        if (use(k)) {
#pragma unroll
            for (int j = 0; j < Q; ++j) {
                const int m = Tb::M(k, j);
                if (m == 1) acc += x[j];
                else if (m == -1) acc -= x[j];
                else if (m != 0) acc += (float)m * x[j];
            }
        }
        a[k] = acc * coef[k];
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            if (!use(k)) continue;
            const int m = Tb::M(k, q);
            if (m == 1) acc += a[k];
            else if (m == -1) acc -= a[k];
            else if (m != 0) acc += (float)m * a[k];
        }
        out[q] = acc;
    }
}

template <class L, bool Les>
__device__ __forceinline__ void collide_dev(const float* d, float* out, const StepParams& p, int coll, float* mac,
                                            const NodeForce* nf, float les_c = 0.f) {
    using Tb = Tables<L>;
    constexpr int Q = L::kQ;
    // a node whose force is exactly zero (every node of a forced level outside the immersed-
    // boundary band, with no constant force) takes the unforced update: the Guo terms vanish
    if (nf && nf->F[0] == 0. && nf->F[1] == 0. && nf->F[2] == 0.) nf = nullptr;
    if constexpr (L::kQ == 19) {
        if (coll == kMrt && !nf && !Les) {
            mrt_d3q19_fused(d, out, p, mac);
            return;
        }
        if (coll == kSrt) {
            if (!nf) {
                srt_d3q19_fused(d, out, p, mac, Les, les_c);
            } else {
                const float F[3] = {(float)nf->F[0], (float)nf->F[1], (float)nf->F[2]};
                srt_d3q19_fused_t<true>(d, out, p, mac, Les, les_c, F);
            }
            return;
        }
    }
    float neq[Q];
    float F[3] = {0.f, 0.f, 0.f};
    if (nf) {
        F[0] = (float)nf->F[0];
        F[1] = (float)nf->F[1];
        F[2] = (float)nf->F[2];
    }
    const float dt = (float)p.dt;
    feq_neq_dev<L>(d, neq, p.scale, p.inv_scale, mac, nf ? F : nullptr, dt);
    float omega = p.omega32;
    if (Les) {
        // non-equilibrium stress (unscaled) and Smagorinsky tau = tau0 + tau_sgs
        float pxx = 0.f, pyy = 0.f, pzz = 0.f, pxy = 0.f, pxz = 0.f, pyz = 0.f;
#pragma unroll
        for (int q = 1; q < Q; ++q) {
            const int cx = Tb::cx(q), cy = Tb::cy(q), cz = Tb::cz(q);
            if (cx) pxx += neq[q];
            if (cy) pyy += neq[q];
            if (cz) pzz += neq[q];
            if (cx * cy) pxy += cx * cy > 0 ? neq[q] : -neq[q];
            if (cx * cz) pxz += cx * cz > 0 ? neq[q] : -neq[q];
            if (cy * cz) pyz += cy * cz > 0 ? neq[q] : -neq[q];
        }
        const float is = p.inv_scale;
        pxx *= is; pyy *= is; pzz *= is; pxy *= is; pxz *= is; pyz *= is;
        if (nf) {
            pxx += dt * F[0] * mac[1];
            pyy += dt * F[1] * mac[2];
            pzz += dt * F[2] * mac[3];
            pxy += 0.5f * dt * (F[0] * mac[1] + F[1] * mac[2]);
            pxz += 0.5f * dt * (F[0] * mac[1] + F[2] * mac[3]);
            pyz += 0.5f * dt * (F[1] * mac[2] + F[2] * mac[3]);
        }
        const float pi2 = pxx * pxx + pyy * pyy + pzz * pzz + 2.f * (pxy * pxy + pxz * pxz + pyz * pyz);
        const float tau0 = (float)p.tau;
        const float tau = tau0 + 0.5f * (sqrtf(tau0 * tau0 + les_c * sqrtf(2.f * pi2)) - tau0);
        omega = 1.f / tau;
    }
    float fq[Q];
    if (nf) {
        // Guo forcing term, scaled to the storage units
        const float ux = mac[1], uy = mac[2], uz = mac[3];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float cx = (float)Tb::cx(q), cy = (float)Tb::cy(q), cz = (float)Tb::cz(q);
            const float cu = signed_dot<L>(q, ux, uy, uz);
            const float cF = signed_dot<L>(q, F[0], F[1], F[2]);
            const float t = 3.f * ((cx - ux) * F[0] + (cy - uy) * F[1] + (cz - uz) * F[2]) + 9.f * cu * cF;
            fq[q] = (float)Tb::w(q) * t * p.scale;
        }
    }
    if (coll == kSrt) {
        const float g = (1.f - 0.5f * omega) * dt;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            out[q] = fmaf(-omega, neq[q], d[q]);
            if (nf) out[q] = fmaf(g, fq[q], out[q]);
        }
        return;
    }
    float lam[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        if (Les) lam[k] = Tb::s(k) > 0. ? ((float)Tb::s(k) - omega) / (float)row_norm2<L>(k) : 0.f;
        else lam[k] = p.mrt_coef[k];
    }
    if constexpr (L::kQ == 19) {
        mrt_d3q19_dev(d, neq, out, omega, lam);
    } else {
        float corr[Q];
        moment_apply<L>(neq, lam, corr, [](int k) { return Tables<L>::s(k) > 0.; });
#pragma unroll
        for (int q = 0; q < Q; ++q) out[q] = fmaf(-omega, neq[q], d[q]) - corr[q];
    }
    if (nf) {
        // With forcing, feq uses the force-shifted velocity, so the momentum of neq is -F dt / 2
        // rather than zero: M^-1 S M neq = omega neq - omega P_conserved(neq) + sum_K ...
        float cc[Q], pc[Q];
#pragma unroll
        for (int k = 0; k < Q; ++k) cc[k] = omega / (float)row_norm2<L>(k);
        moment_apply<L>(neq, cc, pc, [](int k) { return Tables<L>::s(k) == 0.; });
#pragma unroll
        for (int q = 0; q < Q; ++q) out[q] += pc[q];
        // M^-1 (I - S/2) M F = (1 - omega/2) F + (omega/2) P_conserved F - sum_k (s_k - omega)/2 / |M_k|^2 m^F_k M_k
        float coef[Q];
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            const double sk = Tb::s(k);
            coef[k] = sk == 0. ? 0.5f * omega / (float)row_norm2<L>(k)
                    : (sk > 0. ? -0.5f * ((float)sk - omega) / (float)row_norm2<L>(k) : 0.f);
        }
        float src[Q];
        moment_apply<L>(fq, coef, src, [](int k) { return !(Tables<L>::s(k) < 0.); });
        const float g = 1.f - 0.5f * omega;
#pragma unroll
        for (int q = 0; q < Q; ++q) out[q] += dt * fmaf(g, fq[q], src[q]);
    }
}

// ---------------------------------------------------------------- geometry helpers
struct Coord {
    int x[3];  // node coordinates, each in [0, n)
};

__device__ __forceinline__ int wrap_or_ghost(int v, int n, int g, int periodic) {
    // node coordinate v in [-1, n] -> box coordinate
    if (periodic) {
        v = v < 0 ? v + n : (v >= n ? v - n : v);
        return v;
    }
    return v + g;
}

template <class L>
__device__ __forceinline__ bool upstream_missing(const LevelGeom& geo, const Coord& c, int q) {
    using Tb = Tables<L>;
    const int s[3] = {c.x[0] - Tb::cx(q), c.x[1] - Tb::cy(q), c.x[2] - Tb::cz(q)};
#pragma unroll
    for (int a = 0; a < L::kDims; ++a)
        if (!geo.periodic[a] && (s[a] < 0 || s[a] >= geo.n[a])) return true;
    return false;
}

__device__ __forceinline__ int on_faces(const LevelGeom& geo, const Coord& c, int dims) {
    int bits = 0;
    for (int a = 0; a < dims; ++a) {
        if (c.x[a] == 0) bits |= 1 << (2 * a);
        if (c.x[a] == geo.n[a] - 1) bits |= 1 << (2 * a + 1);
    }
    return bits & geo.face_on_box;
}

// Value of the incoming population f(x, q) when its upstream node is missing: the
// bounce-back of the last bounce-back face (in the reference's order xmin, ymin, zmin,
// xmax, ymax, zmax) the node lies on and q enters through, else the stale pre-collision value.
template <class L, class T>
__device__ __forceinline__ T missing_value(int q, int faces, const T* pre, const T* post, const StepParams& p) {
    T v = pre[q];
    if (!p.fuse_bb) return v;
#pragma unroll
    for (int k = 0; k < 2 * L::kDims; ++k) {
        const int face = k < L::kDims ? 2 * k : 2 * (k - L::kDims) + 1;
        if ((faces >> face) & 1) {
            if (p.face_kind[face] == kBcBounceBack && enters_through<L>(q, face)) {
                const int o = bb_source<L>(q, face);
                v = post[o] - (T)(p.bb_term[face][o] * p.scale_d);
            }
        }
    }
    return v;
}

// ---------------------------------------------------------------- the step kernel
// One thread per node of the level box.  Odd selects the layout read (see file comment).
// Bnd: the level has at least one non-periodic axis.  Masked: the box holds absent cells.
// Ext: extended physics compiled in, kExtForce (Guo forcing) and / or kExtLes (Smagorinsky).
// The update of one node c of the level box (collide, stream, stale values / fused bounce back).
template <class L, class S, int Coll, bool Odd, bool Bnd, bool Masked, int Ext>
__device__ __forceinline__ void aa_node(S* __restrict__ f, const LevelGeom& geo, const StepParams& p, const Coord& c) {
    constexpr bool Forced = (Ext & kExtForce) != 0;
    constexpr bool Les = (Ext & kExtLes) != 0;
    using Tb = Tables<L>;
    using St = Storage<S>;
    using T = typename St::T;
    constexpr int Q = L::kQ;

    // box coordinates of x-1, x, x+1 along x and of the node's own row; the rows above and below
    // are formed on the general route only.  Cell indices fit in 32 bits (checked at set-up).
    int bx[3];
#pragma unroll
    for (int d = -1; d <= 1; ++d) bx[d + 1] = wrap_or_ghost(c.x[0] + d, geo.n[0], geo.g[0], geo.periodic[0]);
    const int row_self = geo.a[0] * ((c.x[1] + geo.g[1]) + geo.a[1] * (L::kDims == 3 ? c.x[2] + geo.g[2] : 0));
    const int self = bx[1] + row_self;
    auto cell = [&](int dx, int dy, int dz) -> int {
        const int by = wrap_or_ghost(c.x[1] + dy, geo.n[1], geo.g[1], geo.periodic[1]);
        const int bz = L::kDims == 3 ? wrap_or_ghost(c.x[2] + dz, geo.n[2], geo.g[2], geo.periodic[2]) : 0;
        return bx[dx + 1] + geo.a[0] * (by + geo.a[1] * bz);
    };
    // population planes: uniform 64-bit bases, per-thread 32-bit cell offsets
    const long long st = geo.stride;
    auto plane = [&](int q) -> S* { return f + q * st; };

    // the presence bit is tested once the population loads are issued, so that they do not wait
    // for the info word (an absent cell's slots, and those of its neighbours, are memory of the
    // box like any other: the reads stay in bounds and their values are dropped)
    const uint32_t info = Masked ? __ldg(geo.info + self) : 0u;

    // The node update, given where population q is read from and where its post-collision value goes.
    auto body = [&](auto read_slot, auto write_slot) {
        T pre[Q], post[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) pre[q] = St::load_raw(read_slot(q));
        if (Masked && !(info & kInfoPresent)) return;

        T mac[4];
        NodeForce nf;
        if (Forced) {
            // GetAllForcesForANode (lbm_solver_interface.cpp:132-144): constant force plus node forces;
            // only immersed-boundary stencil nodes (kInfoForce) can hold a node force, the others
            // skip the FP64 read (adding the 0 it would give changes no bit)
            const bool node_force = p.force && (!Masked || (info & kInfoForce));
#pragma unroll
            for (int a = 0; a < 3; ++a) nf.F[a] = p.const_force[a] + (node_force ? p.force[(long long)self * 3 + a] : 0.);
        }
        if constexpr (St::kDeviation) {
            // Smagorinsky constant C: the level's, or 18 c of the learned closure's last evaluation
            const float les_c = Les ? (p.c_node ? 18.f * __ldg(p.c_node + self) : (float)p.les_c) : 0.f;
            collide_dev<L, Les>(pre, post, p, Coll, mac, Forced ? &nf : nullptr, les_c);
        } else {
            collide_exact<L, Les>(pre, post, p, Coll, mac, Forced ? &nf : nullptr);
        }
        if (Masked && (info & kInfoSaveMacro)) {
            double* m = p.macro + (long long)self * 4;
            m[0] = (double)mac[0];
            m[1] = (double)mac[1];
            m[2] = (double)mac[2];
            m[3] = (double)mac[3];
        }

        if (sizeof(S) == 2 && p.sr_seed) {
            // stochastic rounding of the 16-bit stores, one random stream per node
            SrBits rng(sr_seed(p, Odd), (uint32_t)self);
#pragma unroll
            for (int q = 0; q < Q; ++q) St::store_raw_sr(write_slot(q), post[q], rng.next());
        } else {
#pragma unroll
            for (int q = 0; q < Q; ++q) St::store_raw(write_slot(q), post[q]);
        }
        // a masked node with no missing upstream neighbour (bits 1 .. Q-1 clear), or a node of an
        // unmasked box off its non-periodic edges, has nothing to patch
        bool patch = false;
        if (Masked) {
            patch = (info & ((1u << Q) - 2u)) != 0u;
        } else if (Bnd) {
#pragma unroll
            for (int a = 0; a < L::kDims; ++a)
                if (!geo.periodic[a] && (c.x[a] == 0 || c.x[a] == geo.n[a] - 1)) patch = true;
        }
        if (patch) {
            const int faces = Bnd ? (Masked ? (int)((info >> kInfoFaceShift) & 63u) : on_faces(geo, c, L::kDims)) : 0;
#pragma unroll
            for (int q = 1; q < Q; ++q) {
                const bool miss = Masked ? ((info >> q) & 1u) : upstream_missing<L>(geo, c, q);
                if (!miss) continue;
                // off every domain face (coarse/fine interface nodes) the value is the stale one
                const T v = faces ? missing_value<L, T>(q, faces, pre, post, p) : pre[q];
                if (Odd) {
                    St::store_raw(plane(q) + self, v);
                } else {
                    St::store_raw(plane(Tb::opp(q)) + cell(-Tb::cx(q), -Tb::cy(q), -Tb::cz(q)), v);
                }
            }
        }
    };

    // Nodes address their neighbours through three per-thread pointers (cells x-1, x, x+1 of the
    // node's row) plus offsets that are uniform across the launch (plane q and the row step
    // dy a0 + dz a0 a1), unless a periodic y / z row wraps at this node.  Both routes reach the
    // same slots (a ghost frame or an absent cell of a masked box is memory of the box like any
    // other); the uniform one needs no per-access index arithmetic.  The two routes are separate
    // copies of the node update so that each is scheduled on its own.  (Fully periodic full
    // boxes take aa_node_periodic for such rows before reaching here.)
    const bool uniform_rows =
        (!geo.periodic[1] || (c.x[1] > 0 && c.x[1] < geo.n[1] - 1)) &&
        (L::kDims == 2 || !geo.periodic[2] || (c.x[2] > 0 && c.x[2] < geo.n[2] - 1));
    if (uniform_rows) {
        S* const px[3] = {f + (bx[0] + row_self), f + (bx[1] + row_self), f + (bx[2] + row_self)};
        const long long row_y = geo.a[0], row_z = (long long)geo.a[0] * geo.a[1];
        auto uoff = [&](int q, int dy, int dz) -> long long { return q * st + dy * row_y + dz * row_z; };
        body(
            [&](int q) -> S* {
                if (Odd && q != 0) return px[1 - Tb::cx(q)] + uoff(Tb::opp(q), -Tb::cy(q), -Tb::cz(q));
                return px[1] + uoff(q, 0, 0);
            },
            [&](int q) -> S* {
                if (Odd && q != 0) return px[1 + Tb::cx(q)] + uoff(q, Tb::cy(q), Tb::cz(q));
                return px[1] + uoff(Tb::opp(q), 0, 0);
            });
    } else {
        body(
            [&](int q) -> S* {
                if (Odd && q != 0) return plane(Tb::opp(q)) + cell(-Tb::cx(q), -Tb::cy(q), -Tb::cz(q));
                return plane(q) + self;
            },
            [&](int q) -> S* {
                if (Odd && q != 0) return plane(q) + cell(Tb::cx(q), Tb::cy(q), Tb::cz(q));
                return plane(Tb::opp(q)) + self;
            });
    }
}

// The node update on a fully periodic box (no ghost frame) for a node whose rows y +- 1 and
// z +- 1 need no wrap-around: three per-thread pointers (x - 1, x, x + 1 of the node's row, x
// wrapped) plus launch-uniform offsets q * stride + dy a0 + dz a0 a1 reach every slot.
template <class L, class S, int Coll, bool Odd, int Ext>
__device__ __forceinline__ void aa_node_periodic(S* __restrict__ f, const LevelGeom& geo, const StepParams& p,
                                                 const Coord& c) {
    constexpr bool Forced = (Ext & kExtForce) != 0;
    constexpr bool Les = (Ext & kExtLes) != 0;
    using Tb = Tables<L>;
    using St = Storage<S>;
    using T = typename St::T;
    constexpr int Q = L::kQ;
    const int x = c.x[0], n0 = geo.n[0];
    const int xm = x == 0 ? n0 - 1 : x - 1, xp = x == n0 - 1 ? 0 : x + 1;
    const int row = geo.a[0] * (c.x[1] + (L::kDims == 3 ? geo.a[1] * c.x[2] : 0));
    S* const px[3] = {f + (row + xm), f + (row + x), f + (row + xp)};
    const long long st = geo.stride;
    const int a0 = geo.a[0], a01 = geo.a[0] * geo.a[1];
    auto off = [&](int q, int dy, int dz) -> long long { return q * st + (long long)(dy * a0 + dz * a01); };
    T pre[Q], post[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (Odd && q != 0) pre[q] = St::load_raw(px[1 - Tb::cx(q)] + off(Tb::opp(q), -Tb::cy(q), -Tb::cz(q)));
        else pre[q] = St::load_raw(px[1] + off(q, 0, 0));
    }
    T mac[4];
    NodeForce nf;
    if (Forced) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
            nf.F[a] = p.const_force[a] + (p.force ? p.force[(long long)(row + x) * 3 + a] : 0.);
    }
    if constexpr (St::kDeviation) {
        const float les_c = Les ? (p.c_node ? 18.f * __ldg(p.c_node + row + x) : (float)p.les_c) : 0.f;
        collide_dev<L, Les>(pre, post, p, Coll, mac, Forced ? &nf : nullptr, les_c);
    } else {
        collide_exact<L, Les>(pre, post, p, Coll, mac, Forced ? &nf : nullptr);
    }
    if (sizeof(S) == 2 && p.sr_seed) {
        SrBits rng(sr_seed(p, Odd), (uint32_t)(row + x));
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            if (Odd && q != 0) St::store_raw_sr(px[1 + Tb::cx(q)] + off(q, Tb::cy(q), Tb::cz(q)), post[q], rng.next());
            else St::store_raw_sr(px[1] + off(Tb::opp(q), 0, 0), post[q], rng.next());
        }
        return;
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (Odd && q != 0) St::store_raw(px[1 + Tb::cx(q)] + off(q, Tb::cy(q), Tb::cz(q)), post[q]);
        else St::store_raw(px[1] + off(Tb::opp(q), 0, 0), post[q]);
    }
}

// Resident CTAs per SM the register budget is cut for: the plain reduced-precision even step
// (own slots only) fits 64 registers; the odd step and the variants with more state keep 80.
template <class S, bool Odd, bool Bnd, bool Masked, int Ext>
struct StepOccupancy {
    static constexpr int kMinBlocks = (sizeof(S) < 8 && !Odd && !Bnd && !Masked && Ext == 0) ? 4 : 3;
};

template <class L, class S, int Coll, bool Odd, bool Bnd, bool Masked, int Ext = 0>
__global__ void __launch_bounds__(256, (StepOccupancy<S, Odd, Bnd, Masked, Ext>::kMinBlocks))
    aa_step_kernel(S* __restrict__ f, LevelGeom geo, StepParams p) {
    pdl_wait();
    pdl_trigger();
    Coord c;
    if (geo.flat == 2) {
        // the rows' inner nodes first (fn0 divides by n0 - 2), then their two end nodes
        const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x, ni = (uint32_t)geo.n[0] - 2u,
                       inner = ni * (uint32_t)geo.n[1];
        if (t < inner) {
            const uint32_t y = geo.fn0.div(t);
            c.x[0] = 1 + (int)(t - y * ni);
            c.x[1] = (int)y;
        } else {
            const uint32_t k = t - inner;
            c.x[0] = (k & 1u) ? geo.n[0] - 1 : 0;
            c.x[1] = (int)(k >> 1);
        }
    } else if (geo.flat) {
        const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x, y = geo.fn0.div(t);
        c.x[0] = (int)(t - y * (uint32_t)geo.n[0]);
        c.x[1] = (int)y;
    } else {
        c.x[0] = blockIdx.x * blockDim.x + threadIdx.x;
        c.x[1] = blockIdx.y * blockDim.y + threadIdx.y;
    }
    c.x[2] = blockIdx.z + geo.z0;
    if (sizeof(S) == 2 && (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0)
        sr_advance(p, Odd, sr_seed(p, Odd), true);
    if (c.x[0] >= geo.n[0] || c.x[1] >= geo.n[1]) return;
    if constexpr (!Bnd && !Masked) {
        if (c.x[1] > 0 && c.x[1] < geo.n[1] - 1 && (L::kDims == 2 || (c.x[2] > 0 && c.x[2] < geo.n[2] - 1))) {
            aa_node_periodic<L, S, Coll, Odd, Ext>(f, geo, p, c);
            return;
        }
    }
    aa_node<L, S, Coll, Odd, Bnd, Masked, Ext>(f, geo, p, c);
}

// ---------------------------------------------------------------- several levels in one launch

// Levels whose steps follow one another with no transfer between them are independent: one
// persistent launch sweeps all their nodes.  Node i of the batch belongs to the level whose
// [first[l], first[l + 1]) range holds it and is the (i - first[l])-th cell of that box, x fastest;
// each level's range starts at a multiple of the block size, so a block's level is uniform.
// Every level of a multi-level context keeps its info array, so the masked, bounded variant
// (correct for any level) is used throughout; the layout phase is per level.
constexpr int kBatchMax = 8;
constexpr int kBatchThreads = 256;
struct LevelBatch {
    int count;
    int odd[kBatchMax];
    long long first[kBatchMax + 1];
    FastDiv nx[kBatchMax], ny[kBatchMax];  // box extents n0 and n1 of each level
    void* f[kBatchMax];
    LevelGeom geo[kBatchMax];
    const StepParams* params[kBatchMax];  // device copies of the levels' parameters
};

template <class L, class S, int Coll, int Ext>
__global__ void __launch_bounds__(kBatchThreads, 3) aa_batch_kernel(LevelBatch b) {
    const long long total = b.first[b.count];
    for (long long base = (long long)blockIdx.x * kBatchThreads; base < total;
         base += (long long)gridDim.x * kBatchThreads) {
        int l = 0;  // uniform across the block
        while (l + 1 < b.count && base >= b.first[l + 1]) ++l;
        const LevelGeom& geo = b.geo[l];
        if (sizeof(S) == 2 && base == b.first[l] && threadIdx.x == 0)
            sr_advance(*b.params[l], b.odd[l], sr_seed(*b.params[l], b.odd[l]), true);
        const long long k64 = base + threadIdx.x - b.first[l];
        const long long cells = (long long)geo.n[0] * geo.n[1] * geo.n[2];
        if (k64 >= cells) continue;  // padding between two levels' ranges
        const uint32_t k = (uint32_t)k64;  // a level box holds fewer than 2^31 cells
        const uint32_t r = b.nx[l].div(k);
        const uint32_t z = b.ny[l].div(r);
        Coord c;
        c.x[0] = (int)(k - r * (uint32_t)geo.n[0]);
        c.x[1] = (int)(r - z * (uint32_t)geo.n[1]);
        c.x[2] = (int)z;
        S* f = static_cast<S*>(b.f[l]);
        if (b.odd[l]) aa_node<L, S, Coll, true, true, true, Ext>(f, geo, *b.params[l], c);
        else aa_node<L, S, Coll, false, true, true, Ext>(f, geo, *b.params[l], c);
    }
}

// Slot holding the post-stream population f(x, q) in the given layout phase.
template <class L>
__device__ __forceinline__ long long post_stream_slot(const LevelGeom& geo, const Coord& c, int q, bool even_layout) {
    using Tb = Tables<L>;
    int dx = 0, dy = 0, dz = 0, plane = q;
    if (even_layout && q != 0) {
        dx = -Tb::cx(q);
        dy = -Tb::cy(q);
        dz = -Tb::cz(q);
        plane = Tb::opp(q);
    }
    const long long bx = wrap_or_ghost(c.x[0] + dx, geo.n[0], geo.g[0], geo.periodic[0]);
    const long long by = wrap_or_ghost(c.x[1] + dy, geo.n[1], geo.g[1], geo.periodic[1]);
    const long long bz = L::kDims == 3 ? wrap_or_ghost(c.x[2] + dz, geo.n[2], geo.g[2], geo.periodic[2]) : 0;
    return plane * geo.stride + bx + (long long)geo.a[0] * (by + (long long)geo.a[1] * bz);
}

// Slot holding the post-collision population f*(x, o) right after a step whose kernel
// left the given layout: an even step stores it in slot(x, opp(o)), an odd step in slot(x + c_o, o).
template <class L>
__device__ __forceinline__ long long post_collision_slot(const LevelGeom& geo, const Coord& c, int o, bool even_layout) {
    using Tb = Tables<L>;
    int dx = 0, dy = 0, dz = 0, plane = Tb::opp(o);
    if (!even_layout && o != 0) {
        dx = Tb::cx(o);
        dy = Tb::cy(o);
        dz = Tb::cz(o);
        plane = o;
    }
    const long long bx = wrap_or_ghost(c.x[0] + dx, geo.n[0], geo.g[0], geo.periodic[0]);
    const long long by = wrap_or_ghost(c.x[1] + dy, geo.n[1], geo.g[1], geo.periodic[1]);
    const long long bz = L::kDims == 3 ? wrap_or_ghost(c.x[2] + dz, geo.n[2], geo.g[2], geo.periodic[2]) : 0;
    return plane * geo.stride + bx + (long long)geo.a[0] * (by + (long long)geo.a[1] * bz);
}

}  // namespace zl
