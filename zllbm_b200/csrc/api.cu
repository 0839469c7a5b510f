// C ABI of zllbm_b200 (include/zllbm_b200.h): contexts, levels, host exchange, stepping.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <string>
#include <unordered_map>
#include <algorithm>
#include <iterator>
#include <vector>
#include "zllbm_b200.h"
#include "closure_launch.cuh"
#include "topology.cuh"
#include "vtu.cuh"

using namespace zl;

namespace {

struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    ~DeviceBuffer() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    void swap(DeviceBuffer& o) {
        std::swap(ptr, o.ptr);
        std::swap(bytes, o.bytes);
    }
};

struct Level {
    bool active = false;
    LevelGeom geo{};
    LevelMap map{};
    StepParams params{};
    DeviceBuffer f;          // populations
    DeviceBuffer info;       // per-cell info (masked levels only)
    DeviceBuffer mrt64;      // dense M^-1 S M (FP64 storage)
    DeviceBuffer feq_face;   // feq(rho0, U_face) per face, 6 * q doubles
    DeviceBuffer partial;    // conservation partial sums
    int partial_blocks = 0;
    bool bnd = false;        // some axis is not periodic
    bool ordered = false;    // faces applied as ordered passes after the step kernel
    int even_layout = 0;     // 1 after an even step (see aa_kernel.cuh)
    long long nodes = 0;
    long long steps = 0;
    std::vector<uint64_t> codes;  // sorted node codes (kept for multi-level set-ups)
    DeviceBuffer node_codes;      // the codes of zl_set_level_nodes in the caller's order (device)
    long long n_node_codes = 0;
    // coarse/fine transfer with the next coarser level (this level is the fine side)
    DeviceBuffer macro;                                   // rho, u of transfer sources
    DeviceBuffer c2f_target, c2f_offset, c2f_src, c2f_w, c2f_sw32;
    DeviceBuffer c2f_ucell, c2f_ufine, c2f_g;  // distinct sources: cell, kind, values of a transfer
    int n_c2f = 0, n_c2f_src = 0;
    DeviceBuffer f2c_coarse, f2c_fine;
    int n_f2c = 0;
    bool c2f_f2c_disjoint = false;  // no explosion target is a coalescence source: one launch for both
    // the level's immersed-boundary pass may run beside its transfers (zl_advance on level
    // streams): no cell its pass reads lies within two cells of one a transfer writes
    bool ib_concurrent = false;
    long long ib_concurrent_generation = -1;
    bool has_transfer = false;
    double tau_c2f = 0., tau_f2c = 0.;
    // body forces and immersed boundary
    DeviceBuffer force;      // node forces, 3 doubles per cell
    DeviceBuffer mrt64_d;    // M^-1 (I - S/2) M (FP64 forced MRT)
    DeviceBuffer ib_vel;     // node velocities of the forcing pass: x, y, z arrays over the box cells
    DeviceBuffer ib_coord, ib_uvel, ib_area, ib_force, ib_total;
    DeviceBuffer ib_nodes;   // every cell a vertex stencil touches, once
    // the stencils resolved when the vertices are set: per (vertex, stencil node) pair its cell and
    // delta weight; per stencil node the list of its pairs in vertex order (CSR)
    DeviceBuffer ib_pair_cell, ib_pair_w, ib_csr_start, ib_csr_vertex, ib_csr_share;
    int n_vertices = 0, n_ib_nodes = 0;
    int ib_width = 4;        // immersed-boundary stencil: 4 (reference) or 3 (Roma et al.)
    DeviceBuffer c2f_last;   // explosion targets' values at the last transfer (n_c2f x q, storage arithmetic type)
    bool c2f_last_valid = false;
    DeviceBuffer c_node;     // learned closure: c of the last network evaluation per cell
    DeviceBuffer sr_seed;    // stochastic rounding: the two step seeds (StepParams::sr_seed)
    int halo_faces = 0;      // faces whose ghost cells hold a neighbour's slots (zl_set_level_halo)
};

}  // namespace

struct zl_ctx {
    zl_config cfg{};
    int dims = 3;
    int q = 19;
    cudaStream_t stream = nullptr;      // stream all work is issued on
    cudaStream_t own_stream = nullptr;  // the context's own stream
    const LaunchSet* ops = nullptr;
    Level levels[ZL_MAX_LEVELS];
    std::string last_error;
    DeviceBuffer scratch_flag;  // int error flag for kernels that validate codes
    // CUDA graph of two background steps (zl_set_graph)
    bool use_graph = false;
    cudaGraphExec_t graph_exec = nullptr;
    long long graph_generation = -1;
    long long generation = 0;   // bumped by every change of levels, interfaces or vertices
    int graph_layouts = 0;      // bit l: level l's layout when the graph was captured
    DeviceBuffer closure_net;   // zl_mlp of the learned LES closure (zl_set_closure)
    DeviceBuffer closure_err;   // int: a tensor-core wait of the closure step gave up
    int closure_every = 1;      // the network runs on every closure_every-th step of a level
    DeviceBuffer params_dev;    // StepParams of every level on the device (batched steps read them)
    bool batched = true;        // independent consecutive level steps share one launch (zl_set_batching)
    // zl_set_level_streams: zl_advance issues each level's operations on that level's stream,
    // ordered across streams by the levels each operation touches (created on first use)
    bool level_streams = true;
    cudaStream_t lstream[ZL_MAX_LEVELS] = {};
    cudaStream_t ibstream[ZL_MAX_LEVELS] = {};  // immersed-boundary passes beside their level's transfers
    static constexpr int kEvents = 64;
    cudaEvent_t events[kEvents] = {};
    int next_event = 0;
    bool temporal = false;      // time interpolation at the coarse/fine interfaces (zl_set_temporal_interpolation)
    // staging of the node I/O calls (codes, populations, macros): grown on demand and kept until
    // the context is destroyed, so repeated exchanges allocate nothing
    DeviceBuffer stage_codes, stage_data, stage_mac;
};

namespace {

int fail(zl_ctx* ctx, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx) ctx->last_error = buf;
    return code;
}

#define ZL_CUDA(ctx, expr)                                                                          \
    do {                                                                                            \
        cudaError_t _e = (expr);                                                                    \
        if (_e != cudaSuccess)                                                                      \
            return fail(ctx, ZL_EDEVICE, "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e),    \
                        __FILE__, __LINE__);                                                        \
    } while (0)

int alloc(zl_ctx* ctx, DeviceBuffer& b, size_t bytes) {
    b.release();
    if (bytes == 0) return ZL_OK;
    cudaError_t e = cudaMalloc(&b.ptr, bytes);
    if (e != cudaSuccess) {
        b.ptr = nullptr;
        return fail(ctx, ZL_EDEVICE, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    b.bytes = bytes;
    return ZL_OK;
}

// Keep b at least `bytes` large (contents are not preserved when it grows).
int reserve(zl_ctx* ctx, DeviceBuffer& b, size_t bytes) {
    if (b.ptr && b.bytes >= bytes) return ZL_OK;
    return alloc(ctx, b, bytes);
}

double lattice_w(int dims, int q) { return dims == 2 ? Tables<D2Q9>::w(q) : Tables<D3Q19>::w(q); }
int lattice_c(int dims, int q, int a) {
    if (dims == 2) return a == 0 ? Tables<D2Q9>::cx(q) : (a == 1 ? Tables<D2Q9>::cy(q) : 0);
    return a == 0 ? Tables<D3Q19>::cx(q) : (a == 1 ? Tables<D3Q19>::cy(q) : Tables<D3Q19>::cz(q));
}
int lattice_m(int dims, int k, int j) { return dims == 2 ? Tables<D2Q9>::M(k, j) : Tables<D3Q19>::M(k, j); }
double lattice_s(int dims, int k) { return dims == 2 ? Tables<D2Q9>::s(k) : Tables<D3Q19>::s(k); }
int lattice_norm2(int dims, int k) { return dims == 2 ? row_norm2<D2Q9>(k) : row_norm2<D3Q19>(k); }

// feq in the reference's arithmetic order (lbm_solver_interface.cpp:374-417), host side
void host_feq(int dims, double rho, const double* u, double* out) {
    const int q = dims == 2 ? 9 : 19;
    const double uv_sq = dims == 2 ? u[0] * u[0] + u[1] * u[1] : u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    for (int k = 0; k < q; ++k) {
        const double cx = lattice_c(dims, k, 0), cy = lattice_c(dims, k, 1), cz = lattice_c(dims, k, 2);
        const double c_uv = dims == 2 ? u[0] * cx + u[1] * cy : u[0] * cx + u[1] * cy + u[2] * cz;
        out[k] = lattice_w(dims, k) * rho * (1. + 3. * c_uv + 4.5 * c_uv * c_uv - 1.5 * uv_sq);
    }
}

// M^-1 S M (or M^-1 (I - S/2) M) in the reference's loop order
// (collision_model/lbm_collision_model_mrt.cpp:63-107).  M^-1 = M^T diag(1/|M_k|^2).
void host_mrt_matrix(int dims, double relax, bool d_matrix, double* out) {
    const int q = dims == 2 ? 9 : 19;
    std::vector<double> s(q), sm(q * q);
    for (int k = 0; k < q; ++k) {
        const double sk = lattice_s(dims, k);
        s[k] = sk < 0. ? relax : sk;
        if (d_matrix) s[k] = 1. - 0.5 * s[k];
    }
    for (int j = 0; j < q; ++j)
        for (int i = 0; i < q; ++i) {
            double acc = 0.;
            for (int k = 0; k < q; ++k) acc = acc + (i == k ? s[i] : 0.) * (double)lattice_m(dims, k, j);
            sm[i * q + j] = acc;
        }
    for (int j = 0; j < q; ++j)
        for (int i = 0; i < q; ++i) {
            double acc = 0.;
            for (int k = 0; k < q; ++k) {
                const double im = (double)lattice_m(dims, k, i) / (double)lattice_norm2(dims, k);
                acc = acc + im * sm[k * q + j];
            }
            out[i * q + j] = acc;
        }
}

int check_level(zl_ctx* ctx, int level, bool need_active) {
    if (!ctx) return ZL_EINVAL;
    if (level < 0 || level > ctx->cfg.max_level || level >= ZL_MAX_LEVELS)
        return fail(ctx, ZL_EINVAL, "level %d outside [0, %d]", level, ctx->cfg.max_level);
    if (need_active && !ctx->levels[level].active)
        return fail(ctx, ZL_ESTATE, "level %d has no nodes (call zl_set_level_nodes first)", level);
    return ZL_OK;
}

// Copy host codes to a temporary device array.
int upload_codes(zl_ctx* ctx, const uint64_t* codes, int64_t n, DeviceBuffer& d) {
    int rc = reserve(ctx, d, (size_t)n * sizeof(uint64_t));
    if (rc) return rc;
    if (n > 0) ZL_CUDA(ctx, cudaMemcpyAsync(d.ptr, codes, (size_t)n * 8, cudaMemcpyHostToDevice, ctx->stream));
    return ZL_OK;
}

int read_flag(zl_ctx* ctx, int* value) {
    ZL_CUDA(ctx, cudaMemcpyAsync(value, ctx->scratch_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return ZL_OK;
}

int reset_flag(zl_ctx* ctx) {
    ZL_CUDA(ctx, cudaMemsetAsync(ctx->scratch_flag.ptr, 0, sizeof(int), ctx->stream));
    return ZL_OK;
}

}  // namespace

extern "C" {

int zl_abi_version(void) { return ZL_ABI_VERSION; }

int zl_create(const zl_config* config, zl_ctx** out) {
    if (!config || !out) return ZL_EINVAL;
    *out = nullptr;
    if (config->lattice != ZL_D2Q9 && config->lattice != ZL_D3Q19) return ZL_EINVAL;
    if (config->collision != ZL_SRT && config->collision != ZL_MRT) return ZL_EINVAL;
    if (config->storage < ZL_STORAGE_F64 || config->storage > ZL_STORAGE_BF16) return ZL_EINVAL;
    if (config->max_level < 0 || config->max_level >= ZL_MAX_LEVELS) return ZL_EINVAL;
    if (!(config->viscosity > 0.)) return ZL_EINVAL;
    if (config->les < ZL_LES_OFF || config->les > ZL_LES_LEARNED) return ZL_EINVAL;
    if (config->storage_rounding != ZL_ROUND_NEAREST && config->storage_rounding != ZL_ROUND_STOCHASTIC)
        return ZL_EINVAL;
    for (int f = 0; f < 6; ++f)
        if (config->bc_kind[f] < ZL_BC_NONE || config->bc_kind[f] > ZL_BC_CONVECTIVE_OUTFLOW) return ZL_EINVAL;
    const int dims = config->lattice == ZL_D2Q9 ? 2 : 3;
    for (int a = 0; a < dims; ++a) {
        if (config->domain_max[a] <= config->domain_min[a]) return ZL_EINVAL;
        const bool pmin = config->bc_kind[2 * a] == ZL_BC_PERIODIC, pmax = config->bc_kind[2 * a + 1] == ZL_BC_PERIODIC;
        if (pmin != pmax) return ZL_EINVAL;  // periodic faces come in pairs
        for (int f = 2 * a; f < 2 * a + 2; ++f)
            if (config->bc_kind[f] == ZL_BC_CONVECTIVE_OUTFLOW && !(std::fabs(config->bc_velocity[f][a]) > 0.))
                return ZL_EINVAL;  // a convective outflow needs its convection speed
    }
    if (cudaSetDevice(config->device) != cudaSuccess) return ZL_EDEVICE;
    zl_ctx* ctx = new zl_ctx();
    ctx->cfg = *config;
    ctx->dims = dims;
    ctx->q = dims == 2 ? 9 : 19;
    switch (config->storage) {
        case ZL_STORAGE_F64: ctx->ops = &launch_set_f64(); break;
        case ZL_STORAGE_F32: ctx->ops = &launch_set_f32(); break;
        case ZL_STORAGE_F16: ctx->ops = &launch_set_f16(); break;
        default: ctx->ops = &launch_set_bf16(); break;
    }
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return ZL_EDEVICE;
    }
    ctx->stream = ctx->own_stream;
    if (alloc(ctx, ctx->scratch_flag, sizeof(int)) != ZL_OK) {
        cudaStreamDestroy(ctx->own_stream);
        delete ctx;
        return ZL_EDEVICE;
    }
    *out = ctx;
    return ZL_OK;
}

int zl_destroy(zl_ctx* ctx) {
    if (!ctx) return ZL_EINVAL;
    cudaSetDevice(ctx->cfg.device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& l : ctx->levels) {
        l.f.release();
        l.info.release();
        l.mrt64.release();
        l.feq_face.release();
        l.partial.release();
    }
    ctx->scratch_flag.release();
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    for (cudaStream_t& s : ctx->lstream)
        if (s) cudaStreamSynchronize(s), cudaStreamDestroy(s);
    for (cudaStream_t& s : ctx->ibstream)
        if (s) cudaStreamSynchronize(s), cudaStreamDestroy(s);
    for (cudaEvent_t& e : ctx->events)
        if (e) cudaEventDestroy(e);
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return ZL_OK;
}

// Device copy of a level's StepParams (read by the batched multi-level step).
static int sync_params(zl_ctx* ctx, int level) {
    if (!ctx->params_dev.ptr) {
        int rc = alloc(ctx, ctx->params_dev, sizeof(StepParams) * ZL_MAX_LEVELS);
        if (rc) return rc;
    }
    ZL_CUDA(ctx, cudaMemcpy((StepParams*)ctx->params_dev.ptr + level, &ctx->levels[level].params, sizeof(StepParams),
                            cudaMemcpyHostToDevice));
    return ZL_OK;
}

// Level set-up from a node list (codes) or, with codes == nullptr, from the full box whose
// index range is box_mm {min x, min y, min z, max x, max y, max z}.
static int setup_level(zl_ctx* ctx, int level, const uint64_t* codes, int64_t n, const int* box_mm) {
    int rc = check_level(ctx, level, false);
    if (rc) return rc;
    ZL_CUDA(ctx, cudaSetDevice(ctx->cfg.device));
    const int dims = ctx->dims, q = ctx->q;
    Level& L = ctx->levels[level];
    L.active = false;
    L.halo_faces = 0;
    // the vertex set and its node list index the old box
    L.n_vertices = 0;
    L.n_ib_nodes = 0;
    ++ctx->generation;

    DeviceBuffer dcodes, dminmax;
    int mm[6];
    if (codes) {
        if ((rc = upload_codes(ctx, codes, n, dcodes))) return rc;
        if ((rc = alloc(ctx, dminmax, 6 * sizeof(int)))) return rc;
        int init[6] = {INT32_MAX, INT32_MAX, INT32_MAX, 0, 0, 0};
        ZL_CUDA(ctx, cudaMemcpyAsync(dminmax.ptr, init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream));
        ZL_CUDA(ctx, launch_decode_minmax((const uint64_t*)dcodes.ptr, n, dims, (int*)dminmax.ptr, ctx->stream));
        ZL_CUDA(ctx, cudaMemcpyAsync(mm, dminmax.ptr, sizeof(mm), cudaMemcpyDeviceToHost, ctx->stream));
        ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    } else {
        std::memcpy(mm, box_mm, sizeof(mm));
    }

    // Level box.  A periodic axis the level spans completely wraps around (each plane stored
    // once) unless the level also has a non-equilibrium face: the reference then reads its
    // duplicated maximum plane in a face-by-face order that only an explicit copy reproduces,
    // so the duplicate plane is kept and the periodic faces become ordered copy passes.
    LevelGeom geo{};
    LevelMap map{};
    for (int a = 0; a < dims; ++a) {
        const long long dlo = (long long)ctx->cfg.domain_min[a] << level;
        const long long dhi = (long long)ctx->cfg.domain_max[a] << level;
        if (mm[a] < dlo || mm[3 + a] > dhi)
            return fail(ctx, ZL_ETOPOLOGY, "level %d node indices [%d, %d] on axis %d leave the domain [%lld, %lld]",
                        level, mm[a], mm[3 + a], a, dlo, dhi);
    }
    auto make_geo = [&](bool allow_wrap) {
        geo = LevelGeom{};
        map = LevelMap{};
        map.dims = dims;
        for (int a = 0; a < 3; ++a) {
            if (a >= dims) {
                geo.n[a] = 1;
                geo.a[a] = 1;
                map.n[a] = 1;
                continue;
            }
            const long long dlo = (long long)ctx->cfg.domain_min[a] << level;
            const long long dhi = (long long)ctx->cfg.domain_max[a] << level;
            const bool per = ctx->cfg.bc_kind[2 * a] == ZL_BC_PERIODIC;
            if (per && allow_wrap && mm[a] == dlo && mm[3 + a] == dhi) {
                geo.n[a] = (int)(dhi - dlo);
                geo.g[a] = 0;
                geo.periodic[a] = 1;
                map.lo[a] = (int)dlo;
            } else {
                geo.n[a] = mm[3 + a] - mm[a] + 1;
                geo.g[a] = 1;
                geo.periodic[a] = 0;
                map.lo[a] = mm[a];
                if (mm[a] == dlo) geo.face_on_box |= 1 << (2 * a);
                if (mm[3 + a] == dhi) geo.face_on_box |= 1 << (2 * a + 1);
            }
            geo.a[a] = geo.n[a] + 2 * geo.g[a];
            map.n[a] = geo.n[a];
            map.periodic[a] = geo.periodic[a];
        }
    };
    make_geo(true);
    bool has_neq = false, has_conv = false, wraps = false;
    for (int f = 0; f < 2 * dims; ++f) {
        if (ctx->cfg.bc_kind[f] == ZL_BC_NONEQ_EXTRAPOLATION && ((geo.face_on_box >> f) & 1)) has_neq = true;
        if (ctx->cfg.bc_kind[f] == ZL_BC_CONVECTIVE_OUTFLOW && ((geo.face_on_box >> f) & 1)) has_conv = true;
    }
    for (int a = 0; a < dims; ++a) wraps = wraps || geo.periodic[a];
    if (has_neq && wraps) make_geo(false);
    // faces that read their inner neighbour run as passes in the face order, after the step
    L.ordered = has_neq || has_conv;
    const long long cells = (long long)geo.a[0] * geo.a[1] * geo.a[2];
    if (cells >= (1ll << 31) - 64)
        return fail(ctx, ZL_EINVAL, "level %d box of %lld cells exceeds 2^31 (split the level)", level, cells);
    geo.stride = (cells + 63) / 64 * 64;
    geo.fa0 = FastDiv::make((uint32_t)geo.a[0]);
    geo.fa1 = FastDiv::make((uint32_t)geo.a[1]);
    geo.info = nullptr;

    // presence mask; a full box drops it and uses the coordinate-only kernels
    const long long box_nodes = (long long)geo.n[0] * geo.n[1] * geo.n[2];
    // forcing and LES run the extended step variant, which reads the per-cell info array
    const bool need_info = ctx->cfg.max_level > 0 || ctx->cfg.forcing || ctx->cfg.les;
    unsigned long long present = 0;
    if (codes || need_info) {
        if ((rc = alloc(ctx, L.info, (size_t)cells * sizeof(uint32_t)))) return rc;
        ZL_CUDA(ctx, cudaMemsetAsync(L.info.ptr, 0, (size_t)cells * sizeof(uint32_t), ctx->stream));
    }
    if (codes) {
        if ((rc = reset_flag(ctx))) return rc;
        ZL_CUDA(ctx, launch_mark_present((const uint64_t*)dcodes.ptr, n, map, geo, (uint32_t*)L.info.ptr,
                                         (int*)ctx->scratch_flag.ptr, ctx->stream));
        DeviceBuffer dcount;
        if ((rc = alloc(ctx, dcount, sizeof(unsigned long long)))) return rc;
        ZL_CUDA(ctx, cudaMemsetAsync(dcount.ptr, 0, sizeof(unsigned long long), ctx->stream));
        ZL_CUDA(ctx, launch_count_present((const uint32_t*)L.info.ptr, cells, (unsigned long long*)dcount.ptr,
                                          ctx->stream));
        ZL_CUDA(ctx, cudaMemcpyAsync(&present, dcount.ptr, sizeof(present), cudaMemcpyDeviceToHost, ctx->stream));
        int bad = 0;
        if ((rc = read_flag(ctx, &bad))) return rc;
        if (bad) return fail(ctx, ZL_ETOPOLOGY, "level %d: a node code falls outside the level box", level);
    } else {
        present = (unsigned long long)box_nodes;
        if (need_info) ZL_CUDA(ctx, launch_mark_box(geo, (uint32_t*)L.info.ptr, ctx->stream));
    }
    if ((long long)present == box_nodes && !need_info) {
        L.info.release();
    } else {
        geo.info = (const uint32_t*)L.info.ptr;
        launch_node_info(dims, geo, (uint32_t*)L.info.ptr, ctx->stream);
        ZL_CUDA(ctx, cudaGetLastError());
    }
    L.nodes = (long long)present;
    L.bnd = false;
    for (int a = 0; a < dims; ++a)
        if (!geo.periodic[a]) L.bnd = true;

    // parameters (relaxation time per level: lbm_collision_models.cpp:105-118)
    StepParams& p = L.params;
    std::memset(&p, 0, sizeof(p));
    const double dt = 1. / (double)(1u << level);
    p.tau = ctx->cfg.viscosity * 3. / dt + 0.5;
    p.rho0 = ctx->cfg.rho0;
    p.fuse_bb = L.ordered ? 0 : 1;
    p.dt = dt;
    for (int a = 0; a < 3; ++a) p.const_force[a] = ctx->cfg.forcing ? ctx->cfg.constant_force[a] : 0.;
    // FP64 follows the reference, which collides every node with the forcing terms when the
    // solver has forces; the FP32 / FP16 / BF16 step of a level whose forces are all zero (no
    // constant force, no immersed-boundary vertices so far) takes the unforced variant, whose
    // result differs only in rounding (zl_ib_set_vertices switches the level over)
    p.forced = ctx->cfg.forcing && (ctx->cfg.storage == ZL_STORAGE_F64 || p.const_force[0] != 0. ||
                                    p.const_force[1] != 0. || p.const_force[2] != 0.)
                   ? 1
                   : 0;
    p.les = ctx->cfg.les ? 1 : 0;
    {
        const double cs = ctx->cfg.les_cs > 0. ? ctx->cfg.les_cs : 0.16;
        p.les_c = 18. * cs * cs;
    }
    for (int f = 0; f < 6; ++f) {
        p.face_kind[f] = ctx->cfg.bc_kind[f];
        p.conv_u[f] = std::fabs(ctx->cfg.bc_velocity[f][f >> 1]);
    }
    for (int f = 0; f < 2 * dims; ++f) {
        const double* U = ctx->cfg.bc_velocity[f];
        for (int o = 0; o < q; ++o) {
            const double cx = lattice_c(dims, o, 0), cy = lattice_c(dims, o, 1), cz = lattice_c(dims, o, 2);
            const double cu = dims == 2 ? cx * U[0] + cy * U[1] : cx * U[0] + cy * U[1] + cz * U[2];
            p.bb_term[f][o] = 6 * ctx->cfg.rho0 * lattice_w(dims, o) * cu;
        }
    }
    p.omega32 = (float)(1. / p.tau);
    for (int k = 0; k < q; ++k) {
        // fast-path MRT: shear moments relax with 1/tau through the SRT term; the others add
        // (s_k - 1/tau) / |M_k|^2 (conserved moments of neq vanish and stay out)
        const double sk = lattice_s(dims, k);
        p.mrt_coef[k] = sk > 0. ? (float)((sk - 1. / p.tau) / (double)lattice_norm2(dims, k)) : 0.f;
    }
    const double scale = ctx->cfg.storage_scale > 0. ? ctx->cfg.storage_scale : 8192.;
    p.scale = ctx->cfg.storage == ZL_STORAGE_F16 || ctx->cfg.storage == ZL_STORAGE_BF16 ? (float)scale : 1.f;
    p.inv_scale = 1.f / p.scale;
    p.scale_d = (double)p.scale;
    // stochastic rounding of FP16 / BF16 stores: the level's seeds start at 0 with every set-up
    L.sr_seed.release();
    if ((ctx->cfg.storage == ZL_STORAGE_F16 || ctx->cfg.storage == ZL_STORAGE_BF16) &&
        ctx->cfg.storage_rounding == ZL_ROUND_STOCHASTIC) {
        if ((rc = alloc(ctx, L.sr_seed, 2 * sizeof(uint32_t)))) return rc;
        ZL_CUDA(ctx, cudaMemset(L.sr_seed.ptr, 0, 2 * sizeof(uint32_t)));
        p.sr_seed = (uint32_t*)L.sr_seed.ptr;
    }
    if (ctx->cfg.collision == ZL_MRT && ctx->cfg.storage == ZL_STORAGE_F64) {
        std::vector<double> m(q * q);
        host_mrt_matrix(dims, 1. / p.tau, false, m.data());
        if ((rc = alloc(ctx, L.mrt64, m.size() * sizeof(double)))) return rc;
        ZL_CUDA(ctx, cudaMemcpy(L.mrt64.ptr, m.data(), m.size() * sizeof(double), cudaMemcpyHostToDevice));
        p.mrt64 = (const double*)L.mrt64.ptr;
        if (ctx->cfg.forcing) {
            host_mrt_matrix(dims, 1. / p.tau, true, m.data());
            if ((rc = alloc(ctx, L.mrt64_d, m.size() * sizeof(double)))) return rc;
            ZL_CUDA(ctx, cudaMemcpy(L.mrt64_d.ptr, m.data(), m.size() * sizeof(double), cudaMemcpyHostToDevice));
            p.mrt64_d = (const double*)L.mrt64_d.ptr;
        }
    }
    if (ctx->cfg.forcing) {
        if ((rc = alloc(ctx, L.force, (size_t)cells * 3 * sizeof(double)))) return rc;
        ZL_CUDA(ctx, cudaMemset(L.force.ptr, 0, (size_t)cells * 3 * sizeof(double)));
        p.force = (const double*)L.force.ptr;
    }
    std::vector<double> feq_face(6 * q, 0.);
    for (int f = 0; f < 2 * dims; ++f) host_feq(dims, ctx->cfg.rho0, ctx->cfg.bc_velocity[f], &feq_face[f * q]);
    if ((rc = alloc(ctx, L.feq_face, feq_face.size() * sizeof(double)))) return rc;
    ZL_CUDA(ctx, cudaMemcpy(L.feq_face.ptr, feq_face.data(), feq_face.size() * sizeof(double), cudaMemcpyHostToDevice));

    // populations: every slot starts at feq(rho0, default velocity)
    if ((rc = alloc(ctx, L.f, (size_t)q * geo.stride * ctx->ops->elem_bytes))) return rc;
    std::vector<double> f0(q);
    host_feq(dims, ctx->cfg.rho0, ctx->cfg.init_velocity, f0.data());
    if (ctx->cfg.storage != ZL_STORAGE_F64)
        for (int k = 0; k < q; ++k) f0[k] -= lattice_w(dims, k);
    DeviceBuffer dval;
    if ((rc = alloc(ctx, dval, q * sizeof(double)))) return rc;
    ZL_CUDA(ctx, cudaMemcpy(dval.ptr, f0.data(), q * sizeof(double), cudaMemcpyHostToDevice));
    ZL_CUDA(ctx, launch_fill(ctx->cfg.storage, L.f.ptr, geo.stride, q, p, (const double*)dval.ptr, ctx->stream));

    L.partial_blocks = 148 * 4;
    if ((rc = alloc(ctx, L.partial, (size_t)L.partial_blocks * 4 * sizeof(double) + 4 * sizeof(double)))) return rc;

    L.geo = geo;
    L.map = map;
    L.even_layout = 0;
    L.steps = 0;
    L.has_transfer = false;
    L.codes.clear();
    if (ctx->cfg.max_level > 0) {
        if (codes) {
            L.codes.assign(codes, codes + n);
        } else {
            // the box's codes, for the interface look-ups of a multi-level context
            L.codes.reserve((size_t)box_nodes);
            for (int z = mm[2]; z <= (dims == 3 ? mm[5] : mm[2]); ++z)
                for (int y = mm[1]; y <= mm[4]; ++y)
                    for (int x = mm[0]; x <= mm[3]; ++x) {
                        const uint32_t idx[3] = {(uint32_t)x, (uint32_t)y, (uint32_t)z};
                        L.codes.push_back(morton_encode(idx, dims));
                    }
        }
        std::sort(L.codes.begin(), L.codes.end());
        L.codes.erase(std::unique(L.codes.begin(), L.codes.end()), L.codes.end());
    }
    ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if ((rc = sync_params(ctx, level))) return rc;
    // the node list stays on the device for exchanges that pass no codes
    L.node_codes.release();
    L.n_node_codes = 0;
    if (codes) {
        L.node_codes.swap(dcodes);
        L.n_node_codes = n;
    }
    L.active = true;
    return ZL_OK;
}

int zl_set_level_nodes(zl_ctx* ctx, int level, const uint64_t* codes, int64_t n) {
    if (!codes || n <= 0) return fail(ctx, ZL_EINVAL, "empty node set for level %d", level);
    return setup_level(ctx, level, codes, n, nullptr);
}

int zl_set_level_box(zl_ctx* ctx, int level, const int32_t lo[3], const int32_t n[3]) {
    int rc = check_level(ctx, level, false);
    if (rc) return rc;
    if (!lo || !n) return fail(ctx, ZL_EINVAL, "null box");
    int mm[6] = {0, 0, 0, 0, 0, 0};
    for (int a = 0; a < ctx->dims; ++a) {
        if (n[a] < 1 || lo[a] < 0) return fail(ctx, ZL_EINVAL, "box axis %d: lo %d, n %d", a, lo[a], n[a]);
        const long long dlo = (long long)ctx->cfg.domain_min[a] << level;
        const long long dhi = (long long)ctx->cfg.domain_max[a] << level;
        const bool wraps = ctx->cfg.bc_kind[2 * a] == ZL_BC_PERIODIC && lo[a] == dlo && lo[a] + (long long)n[a] == dhi;
        mm[a] = lo[a];
        // a periodic box spanning the domain reads like a node list with the duplicated max plane
        const long long hi = wraps ? dhi : (long long)lo[a] + n[a] - 1;
        if (hi > INT32_MAX) return fail(ctx, ZL_EINVAL, "box axis %d too large", a);
        mm[3 + a] = (int)hi;
    }
    return setup_level(ctx, level, nullptr, 0, mm);
}

static int exchange(zl_ctx* ctx, int level, const uint64_t* codes, double* f_host, double* rho, double* u, int64_t n,
                    bool write) {
    int rc = check_level(ctx, level, true);
    if (rc) return rc;
    if (n < 0) return fail(ctx, ZL_EINVAL, "bad node count");
    if (n == 0) return ZL_OK;
    ZL_CUDA(ctx, cudaSetDevice(ctx->cfg.device));
    Level& L = ctx->levels[level];
    const int q = ctx->q, dims = ctx->dims;
    DeviceBuffer& dbuf = ctx->stage_data;
    DeviceBuffer& dmac = ctx->stage_mac;
    // no codes: the level's own node list (zl_set_level_nodes order), already on the device
    const uint64_t* dcodes = nullptr;
    if (codes) {
        if ((rc = upload_codes(ctx, codes, n, ctx->stage_codes))) return rc;
        dcodes = (const uint64_t*)ctx->stage_codes.ptr;
    } else {
        if (n != L.n_node_codes)
            return fail(ctx, ZL_EINVAL, "level %d: without codes, n must be the %lld nodes given to zl_set_level_nodes",
                        level, L.n_node_codes);
        dcodes = (const uint64_t*)L.node_codes.ptr;
    }
    if ((rc = reset_flag(ctx))) return rc;
    if (write) {
        if ((rc = reserve(ctx, dbuf, (size_t)n * q * sizeof(double)))) return rc;
        ZL_CUDA(ctx, cudaMemcpyAsync(dbuf.ptr, f_host, (size_t)n * q * 8, cudaMemcpyHostToDevice, ctx->stream));
        ZL_CUDA(ctx, ctx->ops->scatter(dims, L.f.ptr, L.geo, L.params, L.map, L.even_layout,
                                       dcodes, (const double*)dbuf.ptr, n,
                                       (int*)ctx->scratch_flag.ptr, ctx->stream));
    } else {
        if (f_host && (rc = reserve(ctx, dbuf, (size_t)n * q * sizeof(double)))) return rc;
        if (rho && (rc = reserve(ctx, dmac, (size_t)n * (dims + 1) * sizeof(double)))) return rc;
        double* drho = rho ? (double*)dmac.ptr : nullptr;
        double* du = rho ? drho + n : nullptr;
        ZL_CUDA(ctx, ctx->ops->gather(dims, L.f.ptr, L.geo, L.params, L.map, L.even_layout,
                                      dcodes, f_host ? (double*)dbuf.ptr : nullptr, drho, du, n,
                                      (int*)ctx->scratch_flag.ptr, ctx->stream));
        if (f_host)
            ZL_CUDA(ctx, cudaMemcpyAsync(f_host, dbuf.ptr, (size_t)n * q * 8, cudaMemcpyDeviceToHost, ctx->stream));
        if (rho) {
            ZL_CUDA(ctx, cudaMemcpyAsync(rho, drho, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream));
            if (u) ZL_CUDA(ctx, cudaMemcpyAsync(u, du, (size_t)n * dims * 8, cudaMemcpyDeviceToHost, ctx->stream));
        }
    }
    int bad = 0;
    if ((rc = read_flag(ctx, &bad))) return rc;
    if (bad) return fail(ctx, ZL_ETOPOLOGY, "level %d: a node code is not part of the level", level);
    return ZL_OK;
}

int zl_set_populations(zl_ctx* ctx, int level, const uint64_t* codes, const double* f, int64_t n) {
    if (n > 0 && !f) return ZL_EINVAL;
    return exchange(ctx, level, codes, const_cast<double*>(f), nullptr, nullptr, n, true);
}

int zl_get_populations(zl_ctx* ctx, int level, const uint64_t* codes, double* f, int64_t n) {
    if (n > 0 && !f) return ZL_EINVAL;
    return exchange(ctx, level, codes, f, nullptr, nullptr, n, false);
}

int zl_get_macros(zl_ctx* ctx, int level, const uint64_t* codes, double* rho, double* u, int64_t n) {
    if (n > 0 && !rho) return ZL_EINVAL;
    return exchange(ctx, level, codes, nullptr, rho, u, n, false);
}

static int ib_pass(zl_ctx* ctx, Level& L, int level);
static int level_faces(zl_ctx* ctx, Level& L);

static int step_level_body(zl_ctx* ctx, int level, bool with_ib);

int zl_step_level(zl_ctx* ctx, int level) {
    int rc = check_level(ctx, level, true);
    if (rc) return rc;
    return step_level_body(ctx, level, true);
}

// The step of a level (its immersed-boundary pass first when with_ib), then its face passes.
static int step_level_body(zl_ctx* ctx, int level, bool with_ib) {
    int rc;
    Level& L = ctx->levels[level];
    if (with_ib && L.n_vertices > 0 && (rc = ib_pass(ctx, L, level))) return rc;
    const bool odd = L.even_layout == 1;
    if (ctx->cfg.les == ZL_LES_LEARNED && ctx->closure_net.ptr) {
        // the network runs inside the collision of a full periodic D3Q19 box
        if (ctx->dims != 3 || ctx->cfg.storage == ZL_STORAGE_F64 || L.bnd || ctx->cfg.forcing ||
            L.nodes != (long long)L.geo.n[0] * L.geo.n[1] * L.geo.n[2])
            return fail(ctx, ZL_EINVAL, "the learned closure runs on full periodic D3Q19 boxes, unforced, "
                                        "in FP32/FP16/BF16 storage");
        const long long cells = (long long)L.geo.a[0] * L.geo.a[1] * L.geo.a[2];
        if (ctx->closure_every > 1 && L.c_node.bytes != (size_t)cells * sizeof(float)) {
            if ((rc = alloc(ctx, L.c_node, (size_t)cells * sizeof(float)))) return rc;
        }
        if (ctx->closure_every <= 1 || L.steps % ctx->closure_every == 0) {
            ZL_CUDA(ctx, closure_learned_step(ctx->cfg.storage, ctx->cfg.collision, odd, L.f.ptr, L.geo, L.params,
                                              (const float*)ctx->closure_net.ptr, (float)(L.params.les_c / 18.),
                                              ctx->closure_every > 1 ? (float*)L.c_node.ptr : nullptr,
                                              (int*)ctx->closure_err.ptr, ctx->stream));
        } else {
            // steps in between reuse each node's c in the Smagorinsky step kernel
            StepParams p = L.params;
            p.c_node = (const float*)L.c_node.ptr;
            ZL_CUDA(ctx, ctx->ops->step(ctx->dims, ctx->cfg.collision, odd, L.bnd, L.geo.info != nullptr, L.f.ptr,
                                        L.geo, p, ctx->stream));
        }
    } else {
        ZL_CUDA(ctx, ctx->ops->step(ctx->dims, ctx->cfg.collision, odd, L.bnd, L.geo.info != nullptr, L.f.ptr,
                                    L.geo, L.params, ctx->stream));
    }
    L.even_layout ^= 1;
    if ((rc = level_faces(ctx, L))) return rc;
    ++L.steps;
    return ZL_OK;
}

int zl_step_level_planes(zl_ctx* ctx, int level, int first, int count, int finish) {
    int rc = check_level(ctx, level, true);
    if (rc) return rc;
    Level& L = ctx->levels[level];
    if (ctx->dims != 3 || L.ordered || L.n_vertices > 0 || ctx->cfg.les == ZL_LES_LEARNED)
        return fail(ctx, ZL_EINVAL,
                    "plane-range steps need a D3Q19 level without ordered face passes, immersed boundary "
                    "or learned closure");
    if (first < 0 || count < 0 || first + count > L.geo.n[2])
        return fail(ctx, ZL_EINVAL, "planes [%d, %d) outside the level's %d", first, first + count, L.geo.n[2]);
    if (count > 0) {
        LevelGeom g = L.geo;
        g.z0 = first;
        g.zn = count;
        ZL_CUDA(ctx, ctx->ops->step(ctx->dims, ctx->cfg.collision, L.even_layout == 1, L.bnd, L.geo.info != nullptr,
                                    L.f.ptr, g, L.params, ctx->stream));
    }
    if (finish) {
        L.even_layout ^= 1;
        if ((rc = level_faces(ctx, L))) return rc;
        ++L.steps;
    }
    return ZL_OK;
}

// Domain faces after a level's step, in the reference's order xmin, ymin, zmin, xmax, ymax, zmax
// (lbm_grid_interface.cpp:225-314); bounce back is fused into the step kernel unless the level
// needs every face as an ordered pass.
static int level_faces(zl_ctx* ctx, Level& L) {
    for (int k = 0; k < 2 * ctx->dims; ++k) {
        const int face = k < ctx->dims ? 2 * k : 2 * (k - ctx->dims) + 1;
        if (!((L.geo.face_on_box >> face) & 1)) continue;
        const int kind = ctx->cfg.bc_kind[face];
        if (kind == ZL_BC_NONEQ_EXTRAPOLATION) {
            ZL_CUDA(ctx, ctx->ops->neq(ctx->dims, L.f.ptr, L.geo, L.params, face, L.even_layout,
                                       (const double*)L.feq_face.ptr + face * ctx->q, ctx->stream));
        } else if (L.ordered && kind == ZL_BC_PERIODIC) {
            // copies need the opposite face on the same level (lbm_periodic.cpp:124-131 skips otherwise)
            const int both = 3 << (2 * (face >> 1));
            if ((L.geo.face_on_box & both) != both) continue;
            ZL_CUDA(ctx, ctx->ops->face(ctx->dims, kind, L.f.ptr, L.geo, L.params, face, L.even_layout, ctx->stream));
        } else if (L.ordered && kind == ZL_BC_BOUNCE_BACK) {
            ZL_CUDA(ctx, ctx->ops->face(ctx->dims, kind, L.f.ptr, L.geo, L.params, face, L.even_layout, ctx->stream));
        } else if (kind == ZL_BC_CONVECTIVE_OUTFLOW) {
            ZL_CUDA(ctx, ctx->ops->face(ctx->dims, kind, L.f.ptr, L.geo, L.params, face, L.even_layout, ctx->stream));
        }
    }
    return ZL_OK;
}

static C2FStencil c2f_stencil(const Level& F) {
    return C2FStencil{(const int*)F.c2f_target.ptr, (const int*)F.c2f_offset.ptr, (const int*)F.c2f_src.ptr,
                      (const double*)F.c2f_w.ptr,      (const int2*)F.c2f_sw32.ptr, F.n_c2f,
                      (const int*)F.c2f_ucell.ptr,     (const uint8_t*)F.c2f_ufine.ptr,
                      F.n_c2f_src,                     F.c2f_g.ptr};
}

// Explosion targets of fine_level <- 0.5 (values at the last transfer + values from the coarse
// level's current state); with save_only, only record the current values as "last".
static int interpolate_interface(zl_ctx* ctx, int fine_level, bool save_only) {
    Level& F = ctx->levels[fine_level];
    Level& C = ctx->levels[fine_level - 1];
    if (!F.has_transfer) return fail(ctx, ZL_ESTATE, "level %d: call zl_set_level_interface first", fine_level);
    if (!save_only && !F.c2f_last_valid)
        return fail(ctx, ZL_ESTATE, "level %d: no transfer yet to interpolate from", fine_level);
    const C2FStencil st = c2f_stencil(F);
    ZL_CUDA(ctx, ctx->ops->c2f(ctx->dims, F.f.ptr, F.geo, F.even_layout, C.f.ptr, C.geo, C.even_layout, F.params,
                               C.params, st, F.tau_c2f, save_only ? F.c2f_last.ptr : nullptr,
                               save_only ? nullptr : F.c2f_last.ptr, save_only ? 0 : 1, nullptr, ctx->stream));
    if (save_only) F.c2f_last_valid = true;
    return ZL_OK;
}

int zl_transfer_levels(zl_ctx* ctx, int fine_level) {
    int rc = check_level(ctx, fine_level, true);
    if (rc) return rc;
    if (fine_level < 1) return fail(ctx, ZL_EINVAL, "level %d has no coarser level", fine_level);
    Level& F = ctx->levels[fine_level];
    Level& C = ctx->levels[fine_level - 1];
    if (!F.has_transfer) return fail(ctx, ZL_ESTATE, "level %d: call zl_set_level_interface first", fine_level);
    const C2FStencil st = c2f_stencil(F);
    const F2CJob job{(const int*)F.f2c_coarse.ptr, (const int*)F.f2c_fine.ptr, F.n_f2c, (const double*)F.macro.ptr,
                     F.tau_f2c};
    const bool fused = F.c2f_f2c_disjoint && F.n_f2c > 0;
    ZL_CUDA(ctx, ctx->ops->c2f(ctx->dims, F.f.ptr, F.geo, F.even_layout, C.f.ptr, C.geo, C.even_layout, F.params,
                               C.params, st, F.tau_c2f, F.c2f_last.ptr, nullptr, 1, fused ? &job : nullptr,
                               ctx->stream));
    F.c2f_last_valid = F.c2f_last.ptr != nullptr;
    if (!fused)
        ZL_CUDA(ctx, ctx->ops->f2c(ctx->dims, F.f.ptr, F.geo, F.even_layout, C.f.ptr, C.geo, C.even_layout, F.params,
                                   C.params, job, ctx->stream));
    return ZL_OK;
}

// Sub-cycled order of one background step (MultiTimeSteppingC2F, amr_project/grid/grid_manager.cpp:997-1023):
// level l is followed by two sweeps of level l + 1.
static void time_stepping_order(int level, int max_level, std::vector<int>* order) {
    order->push_back(level);
    if (level < max_level) {
        time_stepping_order(level + 1, max_level, order);
        time_stepping_order(level + 1, max_level, order);
    }
}

// Steps of several levels with no transfer between them touch disjoint data: one launch of the
// batched kernel covers them (immersed-boundary passes before it, face passes after it, each in
// the levels' order).
static int step_group(zl_ctx* ctx, const std::vector<int>& group) {
    if (group.size() == 1) return zl_step_level(ctx, group[0]);
    // one variant per launch: levels with and without forcing terms step one by one
    int forced = 0, unforced = 0;
    for (int l : group) (ctx->levels[l].params.forced ? forced : unforced) = 1;
    if (forced && unforced) {
        for (int l : group) {
            const int rc = zl_step_level(ctx, l);
            if (rc) return rc;
        }
        return ZL_OK;
    }
    LevelBatch b{};
    b.count = (int)group.size();
    b.first[0] = 0;
    int rc;
    for (size_t i = 0; i < group.size(); ++i) {
        const int l = group[i];
        if ((rc = check_level(ctx, l, true))) return rc;
        Level& L = ctx->levels[l];
        if (L.n_vertices > 0 && (rc = ib_pass(ctx, L, l))) return rc;
        b.odd[i] = L.even_layout == 1;
        b.f[i] = L.f.ptr;
        b.geo[i] = L.geo;
        b.params[i] = (const StepParams*)ctx->params_dev.ptr + l;
        b.nx[i] = FastDiv::make((uint32_t)L.geo.n[0]);
        b.ny[i] = FastDiv::make((uint32_t)L.geo.n[1]);
        // each level's range starts on a block boundary (a block's level is uniform)
        const long long cells = (long long)L.geo.n[0] * L.geo.n[1] * L.geo.n[2];
        b.first[i + 1] = b.first[i] + (cells + kBatchThreads - 1) / kBatchThreads * kBatchThreads;
    }
    const int ext = (forced ? kExtForce : 0) | (ctx->cfg.les ? kExtLes : 0);
    ZL_CUDA(ctx, ctx->ops->batch(ctx->dims, ctx->cfg.collision, ext, b, ctx->stream));
    for (int l : group) {
        Level& L = ctx->levels[l];
        L.even_layout ^= 1;
        if ((rc = level_faces(ctx, L))) return rc;
        ++L.steps;
    }
    return ZL_OK;
}

static bool batchable(const zl_ctx* ctx) {
    if (!ctx->batched || ctx->cfg.max_level == 0 || ctx->cfg.les == ZL_LES_LEARNED) return false;
    for (int l = 0; l <= ctx->cfg.max_level; ++l)
        if (!ctx->levels[l].active || !ctx->levels[l].geo.info) return false;
    return true;
}

namespace {

// Box coordinates of a cell (x fastest).
__device__ __forceinline__ void box_coords(const LevelGeom& geo, int cell, int* b) {
    const uint32_t u = (uint32_t)cell, rest = geo.fa0.div(u), bz = geo.fa1.div(rest);
    b[0] = (int)(u - rest * (uint32_t)geo.a[0]);
    b[1] = (int)(rest - bz * (uint32_t)geo.a[1]);
    b[2] = (int)bz;
}

// Mark every cell within Chebyshev distance 2 of the listed cells (periodic axes wrap).
__global__ void mark_near_kernel(LevelGeom geo, int dims, const int* __restrict__ cells, int n, uint8_t* mark) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int b[3];
    box_coords(geo, cells[t], b);
    const int r2 = dims == 3 ? 2 : 0;
    for (int dz = -r2; dz <= r2; ++dz)
        for (int dy = -2; dy <= 2; ++dy)
            for (int dx = -2; dx <= 2; ++dx) {
                const int d[3] = {dx, dy, dz};
                int c[3];
                bool in = true;
                for (int a = 0; a < 3; ++a) {
                    c[a] = b[a] + d[a];
                    if (geo.periodic[a]) c[a] = c[a] < 0 ? c[a] + geo.a[a] : (c[a] >= geo.a[a] ? c[a] - geo.a[a] : c[a]);
                    in = in && c[a] >= 0 && c[a] < geo.a[a];
                }
                if (in) mark[c[0] + (long long)geo.a[0] * (c[1] + (long long)geo.a[1] * c[2])] = 1;
            }
}

__global__ void any_marked_kernel(const int* __restrict__ cells, int n, const uint8_t* __restrict__ mark, int* flag) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n && mark[cells[t]]) atomicExch(flag, 1);
}

}  // namespace

// Whether each level's immersed-boundary pass may overlap its transfers: the pass reads the
// populations of its stencil nodes (slots of the node and its neighbours) and writes only forces;
// the explosion into this level writes its targets (and their neighbours' slots), the coalescence
// from the next finer level writes coarse nodes of this level.  With every stencil node more than
// two cells from every such node the two touch disjoint data.  Recomputed after any change of
// levels, interfaces or vertices (outside graph capture).
static int refresh_ib_concurrency(zl_ctx* ctx) {
    int rc;
    for (int l = 0; l <= ctx->cfg.max_level; ++l) {
        Level& L = ctx->levels[l];
        if (L.n_vertices <= 0 || L.n_ib_nodes <= 0) {
            L.ib_concurrent = false;
            continue;
        }
        if (L.ib_concurrent_generation == ctx->generation) continue;
        const long long cells = (long long)L.geo.a[0] * L.geo.a[1] * L.geo.a[2];
        DeviceBuffer mark;
        if ((rc = alloc(ctx, mark, (size_t)cells))) return rc;
        ZL_CUDA(ctx, cudaMemsetAsync(mark.ptr, 0, (size_t)cells, ctx->stream));
        mark_near_kernel<<<(L.n_ib_nodes + 127) / 128, 128, 0, ctx->stream>>>(L.geo, ctx->dims, (const int*)L.ib_nodes.ptr,
                                                                            L.n_ib_nodes, (uint8_t*)mark.ptr);
        if ((rc = reset_flag(ctx))) return rc;
        if (l >= 1 && L.has_transfer && L.n_c2f > 0)
            any_marked_kernel<<<(L.n_c2f + 127) / 128, 128, 0, ctx->stream>>>(
                (const int*)L.c2f_target.ptr, L.n_c2f, (const uint8_t*)mark.ptr, (int*)ctx->scratch_flag.ptr);
        if (l < ctx->cfg.max_level && ctx->levels[l + 1].has_transfer && ctx->levels[l + 1].n_f2c > 0) {
            const Level& F = ctx->levels[l + 1];
            any_marked_kernel<<<(F.n_f2c + 127) / 128, 128, 0, ctx->stream>>>(
                (const int*)F.f2c_coarse.ptr, F.n_f2c, (const uint8_t*)mark.ptr, (int*)ctx->scratch_flag.ptr);
        }
        ZL_CUDA(ctx, cudaGetLastError());
        int hit = 0;
        if ((rc = read_flag(ctx, &hit))) return rc;
        L.ib_concurrent = hit == 0;
        L.ib_concurrent_generation = ctx->generation;
    }
    return ZL_OK;
}

static int cuda_wait(zl_ctx* ctx, cudaStream_t s, cudaEvent_t e) {
    ZL_CUDA(ctx, cudaStreamWaitEvent(s, e, 0));
    return ZL_OK;
}
static int cuda_record(zl_ctx* ctx, cudaEvent_t e, cudaStream_t s) {
    ZL_CUDA(ctx, cudaEventRecord(e, s));
    return ZL_OK;
}

// Level streams of zl_advance: one stream per level (finer levels at higher priority: their chains
// of short launches are the critical path), created on first use, and a pool of events.
static int ensure_level_streams(zl_ctx* ctx) {
    if (ctx->lstream[0]) return ZL_OK;
    int least = 0, greatest = 0;
    ZL_CUDA(ctx, cudaDeviceGetStreamPriorityRange(&least, &greatest));
    for (int l = 0; l <= ctx->cfg.max_level; ++l) {
        const int prio = least - l < greatest ? greatest : least - l;
        ZL_CUDA(ctx, cudaStreamCreateWithPriority(&ctx->lstream[l], cudaStreamNonBlocking, prio));
        ZL_CUDA(ctx, cudaStreamCreateWithPriority(&ctx->ibstream[l], cudaStreamNonBlocking, prio));
    }
    for (cudaEvent_t& e : ctx->events) ZL_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return ZL_OK;
}

// The sub-cycled order with every operation on the stream of the level it advances.  An operation
// touches a set of levels (a step or immersed-boundary pass: its level; a transfer: the fine level
// and the coarse one); it waits for the last operation that touched any of them, so operations on
// disjoint levels (the background step and the fine levels' chains of steps, passes and
// transfers) overlap, while every level sees its operations in the reference's order.  The
// results equal the single-stream order's bit for bit.  Works under stream capture: the waits
// become the captured graph's edges.
static int advance_streams(zl_ctx* ctx, int steps, const std::vector<int>& order) {
    int rc = ensure_level_streams(ctx);
    if (rc) return rc;
    const int nl = ctx->cfg.max_level + 1;
    const cudaStream_t main = ctx->stream;
    auto next_event = [&]() -> cudaEvent_t {
        cudaEvent_t e = ctx->events[ctx->next_event];
        ctx->next_event = (ctx->next_event + 1) % zl_ctx::kEvents;
        return e;
    };
    cudaEvent_t last[ZL_MAX_LEVELS], last_step[ZL_MAX_LEVELS];
    cudaStream_t last_stream[ZL_MAX_LEVELS], last_step_stream[ZL_MAX_LEVELS];
    // streams that joined this call's work (and, under capture, the capture): only they rejoin
    bool lused[ZL_MAX_LEVELS] = {}, ibused[ZL_MAX_LEVELS] = {};
    {
        const cudaEvent_t fork = next_event();
        ZL_CUDA(ctx, cudaEventRecord(fork, main));
        for (int l = 0; l < nl; ++l) {
            last[l] = last_step[l] = fork;
            last_stream[l] = last_step_stream[l] = main;
        }
    }
    // run op on the stream of level `home` after the last operations on levels lo .. hi (and
    // after `also`, when given)
    auto run = [&](int home, int lo, int hi, auto op, cudaEvent_t also = nullptr) -> int {
        const cudaStream_t s = ctx->lstream[home];
        lused[home] = true;
        for (int l = lo; l <= hi; ++l)
            if (last_stream[l] != s) ZL_CUDA(ctx, cudaStreamWaitEvent(s, last[l], 0));
        if (also) ZL_CUDA(ctx, cudaStreamWaitEvent(s, also, 0));
        ctx->stream = s;
        const int r = op();
        ctx->stream = main;
        if (r) return r;
        const cudaEvent_t e = next_event();
        ZL_CUDA(ctx, cudaEventRecord(e, s));
        for (int l = lo; l <= hi; ++l) {
            last[l] = e;
            last_stream[l] = s;
        }
        return ZL_OK;
    };
    for (int s = 0; s < steps && !rc; ++s) {
        int count[ZL_MAX_LEVELS] = {0};
        for (int l : order) {
            ++count[l];
            if (ctx->temporal && l > 0 && count[l] % 2 == 0 &&
                (rc = run(l, l - 1, l, [&] { return interpolate_interface(ctx, l, false); })))
                break;
            Level& L = ctx->levels[l];
            // a level's odd-numbered sub-steps follow its transfer (one after every second step);
            // the even-numbered ones follow its own step only and run their immersed-boundary
            // pass in line on the level's stream, where the launches overlap one another
            const bool after_transfer = l > 0 && count[l] % 2 == 1;
            if (L.ib_concurrent && L.n_vertices > 0 && after_transfer) {
                // the immersed-boundary pass on its own stream after the level's last step only,
                // beside the level's transfer; the step waits for both
                const cudaStream_t s = ctx->ibstream[l];
                ibused[l] = true;
                if (last_step_stream[l] != s && (rc = cuda_wait(ctx, s, last_step[l]))) break;
                ctx->stream = s;
                rc = ib_pass(ctx, L, l);
                ctx->stream = main;
                if (rc) break;
                const cudaEvent_t ib_done = next_event();
                if ((rc = cuda_record(ctx, ib_done, s))) break;
                if ((rc = run(l, l, l, [&] { return step_level_body(ctx, l, false); }, ib_done))) break;
            } else if ((rc = run(l, l, l, [&] { return zl_step_level(ctx, l); }))) {
                break;
            }
            last_step[l] = last[l];
            last_step_stream[l] = last_stream[l];
            // InformationFromGridOfDifferentLevel (lbm_solver_interface.cpp:224-238)
            if (l > 0 && count[l] % 2 == 0 && (rc = run(l, l - 1, l, [&] { return zl_transfer_levels(ctx, l); })))
                break;
        }
    }
    // join every level stream back into the caller's stream (also on failure, so that a capture
    // in progress can end)
    for (int l = 0; l < nl; ++l)
        for (int k = 0; k < 2; ++k) {
            if (!(k ? ibused[l] : lused[l])) continue;
            const cudaEvent_t e = next_event();
            ZL_CUDA(ctx, cudaEventRecord(e, k ? ctx->ibstream[l] : ctx->lstream[l]));
            ZL_CUDA(ctx, cudaStreamWaitEvent(main, e, 0));
        }
    return rc;
}

static int advance_direct(zl_ctx* ctx, int steps, const std::vector<int>& order) {
    if (ctx->level_streams && ctx->cfg.max_level > 0) return advance_streams(ctx, steps, order);
    const bool batch = batchable(ctx);
    std::vector<int> group;
    auto flush = [&]() -> int {
        if (group.empty()) return ZL_OK;
        const int rc = step_group(ctx, group);
        group.clear();
        return rc;
    };
    for (int s = 0; s < steps; ++s) {
        int count[ZL_MAX_LEVELS] = {0};
        for (int l : order) {
            ++count[l];
            int rc;
            // the second sub-step of a pair starts half a coarse step after the last transfer:
            // its explosion targets take the average of that transfer and the coarse state now
            if (ctx->temporal && l > 0 && count[l] % 2 == 0) {
                if ((rc = flush()) || (rc = interpolate_interface(ctx, l, false))) return rc;
            }
            if (!batch) {
                if ((rc = zl_step_level(ctx, l))) return rc;
            } else {
                // a level already in the group depends on its own previous step: start a new group
                if (std::find(group.begin(), group.end(), l) != group.end() && (rc = flush())) return rc;
                group.push_back(l);
            }
            // InformationFromGridOfDifferentLevel (lbm_solver_interface.cpp:224-238)
            if (l > 0 && count[l] % 2 == 0) {
                if ((rc = flush())) return rc;
                if ((rc = zl_transfer_levels(ctx, l))) return rc;
            }
        }
        int rc = flush();
        if (rc) return rc;
    }
    return ZL_OK;
}

int zl_advance(zl_ctx* ctx, int steps) {
    if (!ctx || steps < 0) return ZL_EINVAL;
    std::vector<int> order;
    time_stepping_order(0, ctx->cfg.max_level, &order);
    for (int l = 1; l <= ctx->cfg.max_level; ++l)
        if (!ctx->levels[l].has_transfer)
            return fail(ctx, ZL_ESTATE, "level %d: call zl_set_level_interface before zl_advance", l);
    // time interpolation needs the explosion values of a "last transfer": before the first one,
    // those of the current state (recorded outside any graph capture)
    if (ctx->temporal)
        for (int l = 1; l <= ctx->cfg.max_level; ++l)
            if (!ctx->levels[l].c2f_last_valid) {
                const int rc = interpolate_interface(ctx, l, true);
                if (rc) return rc;
            }
    if (ctx->level_streams && ctx->cfg.max_level > 0) {
        const int rc = refresh_ib_concurrency(ctx);
        if (rc) return rc;
    }
    // a closure evaluated every k-th step repeats with period k, not with the graph's two steps
    const bool periodic_closure = ctx->cfg.les == ZL_LES_LEARNED && ctx->closure_net.ptr && ctx->closure_every > 1;
    if (!ctx->use_graph || steps < 2 || periodic_closure) return advance_direct(ctx, steps, order);
    // Two background steps bring every level back to the same population layout, so one captured
    // graph of two steps replays for any number of pairs.
    // the captured launches bake in every level's current population layout
    int layouts = 0;
    for (int l = 0; l <= ctx->cfg.max_level; ++l) layouts |= ctx->levels[l].even_layout << l;
    if (!ctx->graph_exec || ctx->graph_generation != ctx->generation || ctx->graph_layouts != layouts) {
        if (ctx->graph_exec) {
            cudaGraphExecDestroy(ctx->graph_exec);
            ctx->graph_exec = nullptr;
        }
        cudaGraph_t graph = nullptr;
        long long steps_before[ZL_MAX_LEVELS];
        for (int l = 0; l < ZL_MAX_LEVELS; ++l) steps_before[l] = ctx->levels[l].steps;
        ZL_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = advance_direct(ctx, 2, order);
        const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
        for (int l = 0; l < ZL_MAX_LEVELS; ++l) ctx->levels[l].steps = steps_before[l];
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        ZL_CUDA(ctx, e);
        // capture recorded the launches without running them: the host-side layouts went through
        // two full steps and are back where they started
        const cudaError_t ie = cudaGraphInstantiate(&ctx->graph_exec, graph, 0);
        cudaGraphDestroy(graph);
        ZL_CUDA(ctx, ie);
        ctx->graph_generation = ctx->generation;
        ctx->graph_layouts = layouts;
    }
    for (int s = 0; s + 1 < steps; s += 2) {
        ZL_CUDA(ctx, cudaGraphLaunch(ctx->graph_exec, ctx->stream));
        for (int l : order) ctx->levels[l].steps += 2;
    }
    if (steps % 2) return advance_direct(ctx, 1, order);
    return ZL_OK;
}

int zl_set_temporal_interpolation(zl_ctx* ctx, int enabled) {
    if (!ctx) return ZL_EINVAL;
    ctx->temporal = enabled != 0;
    ++ctx->generation;
    return ZL_OK;
}

int zl_interpolate_interface(zl_ctx* ctx, int fine_level) {
    int rc = check_level(ctx, fine_level, true);
    if (rc) return rc;
    if (fine_level < 1) return fail(ctx, ZL_EINVAL, "level %d has no coarser level", fine_level);
    return interpolate_interface(ctx, fine_level, false);
}

int zl_set_batching(zl_ctx* ctx, int enabled) {
    if (!ctx) return ZL_EINVAL;
    ctx->batched = enabled != 0;
    ++ctx->generation;
    return ZL_OK;
}

int zl_set_level_streams(zl_ctx* ctx, int enabled) {
    if (!ctx) return ZL_EINVAL;
    ctx->level_streams = enabled != 0;
    ++ctx->generation;
    return ZL_OK;
}

int zl_set_graph(zl_ctx* ctx, int enabled) {
    if (!ctx) return ZL_EINVAL;
    ctx->use_graph = enabled != 0;
    return ZL_OK;
}

int zl_set_block(zl_ctx* ctx, int level, int x, int y) {
    int rc = check_level(ctx, level, true);
    if (rc) return rc;
    Level& L = ctx->levels[level];
    static_assert(ZL_BLOCK_ROW == kRowKernelBlockX, "row-kernel marker");
    if (x == ZL_BLOCK_ROW) {
        if (y != 1 && y != 2 && y != 4) return fail(ctx, ZL_EINVAL, "row kernel: %d rows per block", y);
        if (!row_eligible(ctx->dims, L.bnd, L.geo.info != nullptr, L.params, ctx->ops->elem_bytes, L.geo))
            return fail(ctx, ZL_EINVAL,
                        "the row kernel needs a full periodic D3Q19 box in FP16/BF16 storage with 128 or 256 nodes per row");
        L.geo.block[0] = x;
        L.geo.block[1] = y;
        ++ctx->generation;
        return ZL_OK;
    }
    const int ax = std::abs(x);
    if (ax < 32 || ax % 32 || y < 1 || ax * y > 256) return fail(ctx, ZL_EINVAL, "block shape %d x %d", x, y);
    if (x < 0 && !pair_eligible(ctx->dims, L.bnd, L.geo.info != nullptr, L.params, ctx->ops->elem_bytes, L.geo))
        return fail(ctx, ZL_EINVAL, "two nodes per thread needs a full periodic D3Q19 box in reduced storage");
    L.geo.block[0] = x;
    L.geo.block[1] = y;
    ++ctx->generation;
    return ZL_OK;
}

int zl_autotune(zl_ctx* ctx, int level, int trials, int32_t* chosen) {
    int rc = check_level(ctx, level, true);
    if (rc) return rc;
    if (trials < 1) trials = 8;
    Level& L = ctx->levels[level];
    // time the step kernel (both layouts) for candidate block shapes on a copy of the populations
    DeviceBuffer saved;
    if ((rc = alloc(ctx, saved, L.f.bytes))) return rc;
    ZL_CUDA(ctx, cudaMemcpyAsync(saved.ptr, L.f.ptr, L.f.bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    // negative x: two nodes per thread (full periodic D3Q19 boxes in reduced storage only);
    // ZL_BLOCK_ROW: one warp per row (FP16/BF16 boxes with 128- or 256-node rows)
    const int shapes[][2] = {{256, 1}, {128, 2}, {128, 1}, {64, 4}, {64, 2}, {32, 8}, {32, 4},
                             {-128, 1}, {-64, 2}, {-256, 1}, {-64, 1},
                             {ZL_BLOCK_ROW, 4}, {ZL_BLOCK_ROW, 2}, {ZL_BLOCK_ROW, 1}};
    const bool pairs = pair_eligible(ctx->dims, L.bnd, L.geo.info != nullptr, L.params, ctx->ops->elem_bytes, L.geo);
    const bool rows = row_eligible(ctx->dims, L.bnd, L.geo.info != nullptr, L.params, ctx->ops->elem_bytes, L.geo);
    cudaEvent_t t0, t1;
    ZL_CUDA(ctx, cudaEventCreate(&t0));
    ZL_CUDA(ctx, cudaEventCreate(&t1));
    float best = 1e30f;
    int best_i = 0;
    const int nshapes = (int)(sizeof(shapes) / sizeof(shapes[0]));
    for (int i = 0; i < nshapes; ++i) {
        LevelGeom g = L.geo;
        g.block[0] = shapes[i][0];
        g.block[1] = shapes[i][1];
        if (g.block[0] == ZL_BLOCK_ROW) {
            if (!rows) continue;
        } else {
            if (g.block[0] < 0 && !pairs) continue;
            if (std::abs(g.block[0]) > 2 * std::max(32, g.n[0])) continue;
        }
        const bool odd0 = L.even_layout == 1;
        for (int warm = 0; warm < 2; ++warm)
            ZL_CUDA(ctx, ctx->ops->step(ctx->dims, ctx->cfg.collision, odd0 != (warm & 1), L.bnd,
                                        L.geo.info != nullptr, L.f.ptr, g, L.params, ctx->stream));
        ZL_CUDA(ctx, cudaEventRecord(t0, ctx->stream));
        for (int k = 0; k < 2 * trials; ++k)
            ZL_CUDA(ctx, ctx->ops->step(ctx->dims, ctx->cfg.collision, odd0 != (k & 1), L.bnd,
                                        L.geo.info != nullptr, L.f.ptr, g, L.params, ctx->stream));
        ZL_CUDA(ctx, cudaEventRecord(t1, ctx->stream));
        ZL_CUDA(ctx, cudaEventSynchronize(t1));
        float ms = 0.f;
        ZL_CUDA(ctx, cudaEventElapsedTime(&ms, t0, t1));
        if (ms < best) {
            best = ms;
            best_i = i;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    ZL_CUDA(ctx, cudaMemcpyAsync(L.f.ptr, saved.ptr, L.f.bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    L.geo.block[0] = shapes[best_i][0];
    L.geo.block[1] = shapes[best_i][1];
    ++ctx->generation;
    if (chosen) {
        chosen[0] = L.geo.block[0];
        chosen[1] = L.geo.block[1];
    }
    return ZL_OK;
}

}  // extern "C"

namespace {

// cell index of a code on a level box, or -1 when the level has no such node
long long cell_of_code(const Level& L, int dims, uint64_t code) {
    if (!std::binary_search(L.codes.begin(), L.codes.end(), code)) return -1;
    uint32_t idx[3];
    zl::morton_decode(code, dims, idx);
    long long b[3] = {0, 0, 0};
    for (int a = 0; a < dims; ++a) {
        long long v = (long long)idx[a] - L.map.lo[a];
        if (L.map.periodic[a] && v == L.map.n[a]) v = 0;
        if (v < 0 || v >= L.map.n[a]) return -1;
        b[a] = v + L.geo.g[a];
    }
    return b[0] + (long long)L.geo.a[0] * (b[1] + (long long)L.geo.a[1] * b[2]);
}

// Lagrangian coefficients of half length 2 at the mid point (grid/grid_interpolation.cpp:87-112)
void lagrange_mid(double* c) {
    const int len = 2, num = 2 * len, offset = len - 1;
    for (int iy = 0; iy < num; ++iy) {
        c[iy] = 1.;
        const double y = (double)iy;
        for (int ix = 0; ix < num; ++ix) {
            if (iy == ix) continue;
            const double x = (double)ix;
            c[iy] *= (0.5 + offset - x) / (y - x);
        }
    }
}

__global__ void or_bits_kernel(uint32_t* info, const int* cells, int n, uint32_t bits) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) info[cells[i]] |= bits;
}

template <class T>
int upload_vec(zl_ctx* ctx, DeviceBuffer& b, const std::vector<T>& v);

// (source row, FP32 bits of the weight) per explosion entry.
std::vector<int2> packed_src_w32(const std::vector<int>& src, const std::vector<double>& w) {
    std::vector<int2> out(src.size());
    for (size_t k = 0; k < src.size(); ++k) {
        const float f = (float)w[k];
        int bits;
        std::memcpy(&bits, &f, 4);
        out[k] = make_int2(src[k], bits);
    }
    return out;
}

template <class T>
int upload_vec(zl_ctx* ctx, DeviceBuffer& b, const std::vector<T>& v) {
    int rc = alloc(ctx, b, v.size() * sizeof(T));
    if (rc) return rc;
    if (!v.empty()) ZL_CUDA(ctx, cudaMemcpy(b.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return ZL_OK;
}

}  // namespace

extern "C" {

int zl_set_level_interface(zl_ctx* ctx, int level, const uint64_t* c2f_fine, int64_t n_c2f,
                           const uint64_t* f2c_coarse, int64_t n_f2c, const uint64_t* coarse_excluded,
                           int64_t n_excluded) {
    int rc = check_level(ctx, level, true);
    if (rc) return rc;
    if (level < 1) return fail(ctx, ZL_EINVAL, "interfaces belong to levels >= 1");
    if ((rc = check_level(ctx, level - 1, true))) return rc;
    if ((n_c2f > 0 && !c2f_fine) || (n_f2c > 0 && !f2c_coarse) || (n_excluded > 0 && !coarse_excluded) ||
        n_c2f < 0 || n_f2c < 0 || n_excluded < 0)
        return fail(ctx, ZL_EINVAL, "bad interface lists");
    ZL_CUDA(ctx, cudaSetDevice(ctx->cfg.device));
    const int dims = ctx->dims;
    Level& F = ctx->levels[level];
    Level& C = ctx->levels[level - 1];
    std::vector<uint64_t> excluded(coarse_excluded, coarse_excluded + n_excluded);
    std::sort(excluded.begin(), excluded.end());
    std::vector<uint64_t> targets(c2f_fine, c2f_fine + n_c2f);
    std::sort(targets.begin(), targets.end());
    double mid[4], one[4] = {0., 1., 0., 0.};
    lagrange_mid(mid);
    const long long clo[3] = {(long long)ctx->cfg.domain_min[0] << (level - 1),
                              (long long)ctx->cfg.domain_min[1] << (level - 1),
                              (long long)ctx->cfg.domain_min[2] << (level - 1)};
    const long long chi[3] = {(long long)ctx->cfg.domain_max[0] << (level - 1),
                              (long long)ctx->cfg.domain_max[1] << (level - 1),
                              (long long)ctx->cfg.domain_max[2] << (level - 1)};
    std::vector<int> tgt, off(1, 0), src, ucell;
    std::vector<uint8_t> ufine;
    std::vector<double> wts;
    // distinct sources (key: cell * 2 + kind) -> row of the per-transfer source table
    std::unordered_map<long long, int> row_of;
    auto source_row = [&](long long cell, int kind) {
        const auto it = row_of.emplace(cell * 2 + kind, (int)ucell.size());
        if (it.second) {
            ucell.push_back((int)cell);
            ufine.push_back((uint8_t)kind);
        }
        return it.first->second;
    };
    for (int64_t i = 0; i < n_c2f; ++i) {
        const long long tc = cell_of_code(F, dims, c2f_fine[i]);
        if (tc < 0) return fail(ctx, ZL_ETOPOLOGY, "level %d: interpolation target is not a node of the level", level);
        uint32_t fidx[3], cidx[3];
        zl::morton_decode(c2f_fine[i], dims, fidx);
        const uint64_t ccode = c2f_fine[i] >> dims;  // SFBitsetToNLowerLevel(1)
        zl::morton_decode(ccode, dims, cidx);
        const double* coef[3] = {one, one, one};
        for (int a = 0; a < dims; ++a) {
            coef[a] = (fidx[a] & 1u) ? mid : one;
            if ((long long)cidx[a] - 1 < clo[a] || (long long)cidx[a] + 2 > chi[a] || (long long)cidx[a] == clo[a])
                return fail(ctx, ZL_ETOPOLOGY,
                            "level %d: interpolation stencil reaches the domain boundary (not supported)", level);
        }
        const int nz = dims == 3 ? 4 : 1;
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < 4; ++iy)
                for (int ix = 0; ix < 4; ++ix) {
                    const double w = dims == 3 ? coef[0][ix] * coef[1][iy] * coef[2][iz] : coef[0][ix] * coef[1][iy];
                    if (!(std::fabs(w) > 1e-6)) continue;
                    uint32_t r[3] = {cidx[0] + ix - 1, cidx[1] + iy - 1, dims == 3 ? cidx[2] + iz - 1 : 0u};
                    const uint64_t rc_code = zl::morton_encode(r, dims);
                    const long long cc = std::binary_search(excluded.begin(), excluded.end(), rc_code)
                                             ? -1 : cell_of_code(C, dims, rc_code);
                    if (cc >= 0) {
                        src.push_back(source_row(cc, 0));
                    } else {
                        const uint64_t fcode = rc_code << dims;  // SFBitsetToNHigherLevel(1)
                        const long long fc = cell_of_code(F, dims, fcode);
                        if (fc < 0)
                            return fail(ctx, ZL_ETOPOLOGY, "level %d: interpolation source found on neither level",
                                        level);
                        if (std::binary_search(targets.begin(), targets.end(), fcode))
                            return fail(ctx, ZL_ETOPOLOGY,
                                        "level %d: an interpolation source is itself a target (order dependent)",
                                        level);
                        src.push_back(source_row(fc, 1));
                    }
                    wts.push_back(w);
                }
        tgt.push_back((int)tc);
        off.push_back((int)src.size());
    }
    {
        // targets grouped by their number of sources, most first (64, 16, 4 or 1 in 3D; a target's
        // sum does not depend on where it sits in the list): the explosion kernel's warps, which
        // cover consecutive targets, then loop over equal counts instead of the largest of mixed
        // ones, and the blocks with the longest loops start first instead of forming the tail
        const size_t nt = tgt.size();
        std::vector<int> perm(nt);
        for (size_t t = 0; t < nt; ++t) perm[t] = (int)t;
        std::stable_sort(perm.begin(), perm.end(),
                         [&](int a, int b) { return off[a + 1] - off[a] > off[b + 1] - off[b]; });
        std::vector<int> tgt2(nt), off2(1, 0), src2;
        std::vector<double> wts2;
        src2.reserve(src.size());
        wts2.reserve(wts.size());
        for (size_t t = 0; t < nt; ++t) {
            const int p = perm[t];
            tgt2[t] = tgt[p];
            src2.insert(src2.end(), src.begin() + off[p], src.begin() + off[p + 1]);
            wts2.insert(wts2.end(), wts.begin() + off[p], wts.begin() + off[p + 1]);
            off2.push_back((int)src2.size());
        }
        tgt.swap(tgt2);
        off.swap(off2);
        src.swap(src2);
        wts.swap(wts2);
        // source rows grouped by kind (coarse-level sources first, then fine ones): the sources
        // kernel's warps then take one of its two paths
        const size_t ns = ucell.size();
        std::vector<int> row_new(ns), ucell2;
        std::vector<uint8_t> ufine2;
        ucell2.reserve(ns);
        ufine2.reserve(ns);
        for (int kind = 0; kind < 2; ++kind)
            for (size_t r = 0; r < ns; ++r)
                if (ufine[r] == kind) {
                    row_new[r] = (int)ucell2.size();
                    ucell2.push_back(ucell[r]);
                    ufine2.push_back(ufine[r]);
                }
        for (int& r : src) r = row_new[r];
        ucell.swap(ucell2);
        ufine.swap(ufine2);
    }
    std::vector<int> f2c_c, f2c_f;
    for (int64_t i = 0; i < n_f2c; ++i) {
        const long long cc = cell_of_code(C, dims, f2c_coarse[i]);
        const long long fc = cell_of_code(F, dims, f2c_coarse[i] << dims);
        if (cc < 0 || fc < 0)
            return fail(ctx, ZL_ETOPOLOGY, "level %d: coalescence node missing on the fine or coarse level", level);
        f2c_c.push_back((int)cc);
        f2c_f.push_back((int)fc);
    }
    if ((rc = upload_vec(ctx, F.c2f_target, tgt)) || (rc = upload_vec(ctx, F.c2f_offset, off)) ||
        (rc = upload_vec(ctx, F.c2f_src, src)) || (rc = upload_vec(ctx, F.c2f_ucell, ucell)) ||
        (rc = upload_vec(ctx, F.c2f_ufine, ufine)) || (rc = upload_vec(ctx, F.c2f_w, wts)) ||
        (rc = upload_vec(ctx, F.c2f_sw32, packed_src_w32(src, wts))) ||
        (rc = upload_vec(ctx, F.f2c_coarse, f2c_c)) || (rc = upload_vec(ctx, F.f2c_fine, f2c_f)))
        return rc;
    F.n_c2f = (int)tgt.size();
    F.n_c2f_src = (int)ucell.size();
    // source values in the storage's arithmetic type (FP64 for FP64 storage, FP32 otherwise; FP32
    // rows padded to whole groups of four)
    const size_t g_elem = ctx->cfg.storage == ZL_STORAGE_F64 ? sizeof(double) : sizeof(float);
    const size_t g_row = g_elem == sizeof(double) ? (size_t)ctx->q : (size_t)(ctx->q + 3) / 4 * 4;
    if ((rc = alloc(ctx, F.c2f_g, (size_t)std::max(F.n_c2f_src, 1) * g_row * g_elem))) return rc;
    F.n_f2c = (int)f2c_c.size();
    {
        std::vector<int> a(tgt), b(f2c_f);
        std::sort(a.begin(), a.end());
        std::sort(b.begin(), b.end());
        std::vector<int> common;
        std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(common));
        F.c2f_f2c_disjoint = common.empty();
    }
    if ((rc = alloc(ctx, F.c2f_last, (size_t)std::max(F.n_c2f, 1) * ctx->q * g_elem))) return rc;
    F.c2f_last_valid = false;
    // coalescence sources keep rho, u of their last collision
    if (F.n_f2c > 0) {
        const long long cells = (long long)F.geo.a[0] * F.geo.a[1] * F.geo.a[2];
        if ((rc = alloc(ctx, F.macro, (size_t)cells * 4 * sizeof(double)))) return rc;
        ZL_CUDA(ctx, cudaMemset(F.macro.ptr, 0, (size_t)cells * 4 * sizeof(double)));
        F.params.macro = (double*)F.macro.ptr;
        if ((rc = sync_params(ctx, level))) return rc;
        or_bits_kernel<<<(F.n_f2c + 127) / 128, 128, 0, ctx->stream>>>((uint32_t*)F.info.ptr,
                                                                        (const int*)F.f2c_fine.ptr, F.n_f2c,
                                                                        kInfoSaveMacro);
        ZL_CUDA(ctx, cudaGetLastError());
    }
    // relaxation-time ratios (collision_model/lbm_collision_models.cpp:142-151)
    const double vis = ctx->cfg.viscosity;
    const double dt_c = 1. / (double)(1u << (level - 1)), dt_f = 1. / (double)(1u << level);
    {
        const double tf = vis * 3. / dt_c * 2. + 0.5, tc = vis * 3. / dt_c + 0.5;
        F.tau_c2f = 0.5 * tf / tc;  // the coarse level's tau_stream_c2f
    }
    {
        const double tf = vis * 3. / dt_f + 0.5, tc = vis * 3. / dt_f / 2 + 0.5;
        F.tau_f2c = 2. * tc / tf;   // the fine level's tau_stream_f2c
    }
    ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    F.has_transfer = true;
    ++ctx->generation;
    return ZL_OK;
}

int zl_conservation(zl_ctx* ctx, int level, double* out) {
    int rc = check_level(ctx, level, true);
    if (rc) return rc;
    if (!out) return ZL_EINVAL;
    Level& L = ctx->levels[level];
    double* partial = (double*)L.partial.ptr;
    double* result = partial + (size_t)L.partial_blocks * 4;
    ZL_CUDA(ctx, ctx->ops->conservation(ctx->dims, L.f.ptr, L.geo, L.params, L.even_layout, partial,
                                        L.partial_blocks, result, ctx->stream));
    double host[4];
    ZL_CUDA(ctx, cudaMemcpyAsync(host, result, sizeof(host), cudaMemcpyDeviceToHost, ctx->stream));
    ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k <= ctx->dims; ++k) out[k] = host[k];
    for (int k = 0; k <= ctx->dims; ++k)
        if (!std::isfinite(host[k])) return fail(ctx, ZL_ENAN, "non-finite conservation sum on level %d", level);
    return ZL_OK;
}

static IbVertices ib_view(zl_ctx* ctx, Level& L, int level) {
    IbVertices v;
    v.coord = (const double*)L.ib_coord.ptr;
    v.vel = (const double*)L.ib_uvel.ptr;
    v.area = (const double*)L.ib_area.ptr;
    v.force = (double*)L.ib_force.ptr;
    v.n = L.n_vertices;
    v.width = L.ib_width;
    const double dx0 = ctx->cfg.dx > 0. ? ctx->cfg.dx : 1.;
    v.dx = dx0 / (double)(1u << level);
    return v;
}

static int ib_pass(zl_ctx* ctx, Level& L, int level) {
    IbVertices v = ib_view(ctx, L, level);
    ZL_CUDA(ctx, ctx->ops->ib_touch(ctx->dims, L.f.ptr, L.geo, L.params, L.even_layout, (const int*)L.ib_nodes.ptr,
                                    L.n_ib_nodes, (double*)L.ib_vel.ptr, ctx->stream));
    // interpolation: kIbForceLanes lanes per vertex; spread: kIbSpreadLanes lanes per node
    const unsigned threads = kIbForceThreads,
                   blocks = (unsigned)(((long long)v.n * kIbForceLanes + threads - 1) / threads);
    const unsigned nblocks = (unsigned)(((long long)L.n_ib_nodes * kIbSpreadLanes + 127) / 128);
    const int* pc = (const int*)L.ib_pair_cell.ptr;
    const double* pw = (const double*)L.ib_pair_w.ptr;
    const int *cs = (const int*)L.ib_csr_start.ptr, *cv = (const int*)L.ib_csr_vertex.ptr;
    const double* csh = (const double*)L.ib_csr_share.ptr;
    // dependent launches: each kernel's launch overlaps the tail of the one before it
    const double* vel = (const double*)L.ib_vel.ptr;
    const long long cells = (long long)L.geo.a[0] * L.geo.a[1] * L.geo.a[2];
    const int* nodes = (const int*)L.ib_nodes.ptr;
    double* nf = (double*)L.force.ptr;
    if (ctx->dims == 2) {
        ZL_CUDA(ctx, launch_dependent(ib_force_kernel<2>, dim3(blocks), dim3(threads), 0, ctx->stream, v, pc, pw, vel,
                                      cells));
        ZL_CUDA(ctx, launch_dependent(ib_spread_kernel<2>, dim3(nblocks), dim3(128), 0, ctx->stream, v, nodes,
                                      L.n_ib_nodes, cs, cv, csh, nf));
    } else {
        ZL_CUDA(ctx, launch_dependent(ib_force_kernel<3>, dim3(blocks), dim3(threads), 0, ctx->stream, v, pc, pw, vel,
                                      cells));
        ZL_CUDA(ctx, launch_dependent(ib_spread_kernel<3>, dim3(nblocks), dim3(128), 0, ctx->stream, v, nodes,
                                      L.n_ib_nodes, cs, cv, csh, nf));
    }
    return ZL_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- halo faces (slab sharding)
namespace {

// Cells of the plane of `face` at box coordinate `layer` on the face's axis: every cell of the
// two other axes' allocated extents, the lower one fastest.
struct FacePlane {
    int axis, b, c;       // the face's axis and the two others (b fastest)
    int nb, nc;           // allocated extents of b and c
    int layer;            // box coordinate on `axis`
    long long stride[3];  // cell stride per axis
};

FacePlane face_plane(const LevelGeom& geo, int dims, int face, bool ghost) {
    FacePlane fp{};
    fp.axis = face >> 1;
    const bool hi = face & 1;
    int others[2], k = 0;
    for (int a = 0; a < 3; ++a)
        if (a != fp.axis) others[k++] = a;
    fp.b = others[0];
    fp.c = others[1];
    fp.nb = geo.a[fp.b];
    fp.nc = dims == 3 || fp.c < 2 ? geo.a[fp.c] : 1;
    const int g = geo.g[fp.axis], n = geo.n[fp.axis];
    fp.layer = ghost ? (hi ? g + n : g - 1) : (hi ? g + n - 1 : g);
    fp.stride[0] = 1;
    fp.stride[1] = geo.a[0];
    fp.stride[2] = (long long)geo.a[0] * geo.a[1];
    return fp;
}

__global__ void mark_plane_present_kernel(uint32_t* info, FacePlane fp) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)fp.nb * fp.nc) return;
    const long long cell = fp.layer * fp.stride[fp.axis] + (t % fp.nb) * fp.stride[fp.b] + (t / fp.nb) * fp.stride[fp.c];
    info[cell] = kInfoPresent;
}

// Clear the missing-upstream bits (1 .. q - 1) of every cell before they are derived again.
__global__ void clear_missing_kernel(uint32_t* info, long long cells, int q) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t < cells) info[t] &= ~((1u << q) - 2u);
}

// Copy the planes `planes[0 .. np)` of the face plane between the population array and a packed
// buffer [np][nc][nb] of raw storage elements (E bytes each).
template <class E>
__global__ void halo_copy_kernel(E* f, long long stride, FacePlane fp, int np, int4 planes_lo, int4 planes_hi,
                                 E* buf, int pack) {
    pdl_wait();
    pdl_trigger();
    const long long per = (long long)fp.nb * fp.nc;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= per * np) return;
    const int k = (int)(t / per);
    const long long r = t % per;
    const int pl[8] = {planes_lo.x, planes_lo.y, planes_lo.z, planes_lo.w, planes_hi.x, planes_hi.y, planes_hi.z,
                       planes_hi.w};
    const long long cell = fp.layer * fp.stride[fp.axis] + (r % fp.nb) * fp.stride[fp.b] + (r / fp.nb) * fp.stride[fp.c];
    E* slot = f + pl[k] * stride + cell;
    if (pack) buf[t] = *slot;
    else *slot = buf[t];
}

}  // namespace

extern "C" {

// Population planes that cross `face` inward (toward the box) or outward.
static int face_planes(int dims, int face, bool inward, int* planes) {
    const int axis = face >> 1;
    const int sign = (face & 1) ? (inward ? -1 : 1) : (inward ? 1 : -1);
    const int q = dims == 2 ? 9 : 19;
    int n = 0;
    for (int k = 0; k < q; ++k)
        if (lattice_c(dims, k, axis) == sign) planes[n++] = k;
    return n;
}

int zl_set_level_halo(zl_ctx* ctx, int level, int faces) {
    int rc = check_level(ctx, level, true);
    if (rc) return rc;
    Level& L = ctx->levels[level];
    if (faces & ~((1 << (2 * ctx->dims)) - 1)) return fail(ctx, ZL_EINVAL, "halo faces 0x%x", faces);
    for (int f = 0; f < 2 * ctx->dims; ++f) {
        if (!((faces >> f) & 1)) continue;
        if (ctx->cfg.bc_kind[f] != ZL_BC_NONE || !L.geo.g[f >> 1] || !((L.geo.face_on_box >> f) & 1))
            return fail(ctx, ZL_EINVAL, "level %d: a halo face needs ZL_BC_NONE and the level box on the domain face", level);
    }
    if (ctx->cfg.max_level > 0 || ctx->cfg.forcing || ctx->cfg.les == ZL_LES_LEARNED)
        return fail(ctx, ZL_ESTATE, "halo faces are for single-level contexts without forcing");
    ZL_CUDA(ctx, cudaSetDevice(ctx->cfg.device));
    const long long cells = (long long)L.geo.a[0] * L.geo.a[1] * L.geo.a[2];
    if (!L.info.ptr) {
        // a full box gets its per-cell info (presence, missing-upstream and face bits)
        if ((rc = alloc(ctx, L.info, (size_t)cells * sizeof(uint32_t)))) return rc;
        ZL_CUDA(ctx, cudaMemsetAsync(L.info.ptr, 0, (size_t)cells * sizeof(uint32_t), ctx->stream));
        ZL_CUDA(ctx, launch_mark_box(L.geo, (uint32_t*)L.info.ptr, ctx->stream));
        L.geo.info = (const uint32_t*)L.info.ptr;
    }
    // ghost cells of a halo face hold the neighbour's slots: present for the neighbour lookups of
    // the nodes next to them, never stepped themselves
    for (int f = 0; f < 2 * ctx->dims; ++f) {
        if (!((faces >> f) & 1)) continue;
        const FacePlane fp = face_plane(L.geo, ctx->dims, f, true);
        const long long n = (long long)fp.nb * fp.nc;
        mark_plane_present_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>((uint32_t*)L.info.ptr, fp);
    }
    clear_missing_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, ctx->stream>>>((uint32_t*)L.info.ptr, cells, ctx->q);
    launch_node_info(ctx->dims, L.geo, (uint32_t*)L.info.ptr, ctx->stream, L.halo_faces | faces);
    ZL_CUDA(ctx, cudaGetLastError());
    ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    L.halo_faces |= faces;
    // a full box periodic along x and y with both z faces connected: the full-box kernels apply
    const long long box_nodes = (long long)L.geo.n[0] * L.geo.n[1] * L.geo.n[2];
    L.geo.ring = ctx->dims == 3 && L.geo.periodic[0] && L.geo.periodic[1] && (L.halo_faces & 48) == 48 &&
                 L.nodes == box_nodes;
    ++ctx->generation;
    return ZL_OK;
}

int zl_halo_bytes(zl_ctx* ctx, int level, int face, int64_t* bytes) {
    int rc = check_level(ctx, level, true);
    if (rc) return rc;
    if (face < 0 || face >= 2 * ctx->dims || !bytes) return fail(ctx, ZL_EINVAL, "bad halo face");
    const Level& L = ctx->levels[level];
    const FacePlane fp = face_plane(L.geo, ctx->dims, face, true);
    int planes[8];
    const int np = face_planes(ctx->dims, face, true, planes);
    *bytes = (int64_t)np * fp.nb * fp.nc * ctx->ops->elem_bytes;
    return ZL_OK;
}

static int halo_copy(zl_ctx* ctx, int level, int face, int stage, void* buf, bool pack) {
    int rc = check_level(ctx, level, true);
    if (rc) return rc;
    Level& L = ctx->levels[level];
    if (face < 0 || face >= 2 * ctx->dims || !((L.halo_faces >> face) & 1) || (stage != 0 && stage != 1) || !buf)
        return fail(ctx, ZL_EINVAL, "halo copy: face %d is not a halo face of level %d, or bad stage / buffer", face, level);
    // stage 0 (after an even step): the boundary plane's inward planes travel to the neighbour's
    // ghost plane (its outward planes); stage 1 (after an odd step): the ghost plane's outward
    // planes travel back to the neighbour's boundary plane (its inward planes)
    const bool ghost = pack ? stage == 1 : stage == 0;
    const bool inward = pack ? stage == 0 : stage == 1;
    const FacePlane fp = face_plane(L.geo, ctx->dims, face, ghost);
    int planes[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int np = face_planes(ctx->dims, face, inward, planes);
    const long long n = (long long)np * fp.nb * fp.nc;
    const int4 lo = make_int4(planes[0], planes[1], planes[2], planes[3]);
    const int4 hi = make_int4(planes[4], planes[5], planes[6], planes[7]);
    const unsigned blocks = (unsigned)((n + 255) / 256);
    switch (ctx->ops->elem_bytes) {
        case 8:
            ZL_CUDA(ctx, launch_dependent(halo_copy_kernel<uint64_t>, dim3(blocks), dim3(256), 0, ctx->stream,
                                          (uint64_t*)L.f.ptr, L.geo.stride, fp, np, lo, hi, (uint64_t*)buf, pack));
            break;
        case 4:
            ZL_CUDA(ctx, launch_dependent(halo_copy_kernel<uint32_t>, dim3(blocks), dim3(256), 0, ctx->stream,
                                          (uint32_t*)L.f.ptr, L.geo.stride, fp, np, lo, hi, (uint32_t*)buf, pack));
            break;
        default:
            ZL_CUDA(ctx, launch_dependent(halo_copy_kernel<uint16_t>, dim3(blocks), dim3(256), 0, ctx->stream,
                                          (uint16_t*)L.f.ptr, L.geo.stride, fp, np, lo, hi, (uint16_t*)buf, pack));
            break;
    }
    ZL_CUDA(ctx, cudaGetLastError());
    return ZL_OK;
}

int zl_halo_pack(zl_ctx* ctx, int level, int face, int stage, void* buf_device) {
    return halo_copy(ctx, level, face, stage, buf_device, true);
}

int zl_halo_unpack(zl_ctx* ctx, int level, int face, int stage, const void* buf_device) {
    return halo_copy(ctx, level, face, stage, const_cast<void*>(buf_device), false);
}

int zl_ib_set_vertices(zl_ctx* ctx, int level, int64_t n, const double* coordinates, const double* velocity,
                       const double* area) {
    int rc = check_level(ctx, level, true);
    if (rc) return rc;
    if (!ctx->cfg.forcing) return fail(ctx, ZL_ESTATE, "immersed boundaries need config->forcing = 1");
    if (n < 0 || (n > 0 && (!coordinates || !velocity || !area))) return fail(ctx, ZL_EINVAL, "bad vertex arrays");
    Level& L = ctx->levels[level];
    // the level has no vertex set (its pass does not run) unless this call completes
    struct Incomplete {
        Level& L;
        bool done = false;
        ~Incomplete() {
            if (!done) L.n_vertices = 0;
        }
    } guard{L};
    L.n_vertices = 0;
    ++ctx->generation;
    if (n > 0 && !L.params.forced) {
        // node forces from now on: the level's steps take the forced variant
        L.params.forced = 1;
        if ((rc = sync_params(ctx, level))) return rc;
    }
    if ((rc = alloc(ctx, L.ib_coord, (size_t)n * 3 * 8)) || (rc = alloc(ctx, L.ib_uvel, (size_t)n * 3 * 8)) ||
        (rc = alloc(ctx, L.ib_area, (size_t)n * 8)) || (rc = alloc(ctx, L.ib_force, (size_t)n * 3 * 8)) ||
        (rc = alloc(ctx, L.ib_total, 3 * 8)))
        return rc;
    const long long cells = (long long)L.geo.a[0] * L.geo.a[1] * L.geo.a[2];
    if (L.ib_vel.bytes != (size_t)cells * 3 * 8 && (rc = alloc(ctx, L.ib_vel, (size_t)cells * 3 * 8))) return rc;
    if (n > 0) {
        ZL_CUDA(ctx, cudaMemcpy(L.ib_coord.ptr, coordinates, (size_t)n * 3 * 8, cudaMemcpyHostToDevice));
        ZL_CUDA(ctx, cudaMemcpy(L.ib_uvel.ptr, velocity, (size_t)n * 3 * 8, cudaMemcpyHostToDevice));
        ZL_CUDA(ctx, cudaMemcpy(L.ib_area.ptr, area, (size_t)n * 8, cudaMemcpyHostToDevice));
        ZL_CUDA(ctx, cudaMemset(L.ib_force.ptr, 0, (size_t)n * 3 * 8));
    }
    L.n_vertices = (int)n;
    // every stencil node must exist on the level (the reference logs an error otherwise); the
    // distinct stencil cells become the node list of the pass's first launch.  Nodes of the
    // previous list that no new stencil touches drop their force (all of them when the new set
    // is empty or rejected).
    const int old_nodes = L.n_ib_nodes;
    L.n_ib_nodes = 0;
    auto release = [&](const void* mark) -> int {
        if (old_nodes <= 0 || !L.force.ptr) return ZL_OK;
        ib_release_kernel<<<(unsigned)((old_nodes + 255) / 256), 256, 0, ctx->stream>>>(
            (const int*)L.ib_nodes.ptr, old_nodes, (const uint32_t*)mark, (double*)L.force.ptr);
        ZL_CUDA(ctx, cudaGetLastError());
        return ZL_OK;
    };
    if (n == 0 && (rc = release(nullptr))) return rc;
    if (n > 0) {
        IbVertices v = ib_view(ctx, L, level);
        if ((rc = reset_flag(ctx))) return rc;
        if (cells > 0x7fffffffll) return fail(ctx, ZL_ETOOLARGE, "level %d: box too large for the node list", level);
        DeviceBuffer mark, sel, count, tmp;
        if ((rc = alloc(ctx, mark, (size_t)cells * 4)) || (rc = alloc(ctx, sel, (size_t)cells * 4)) ||
            (rc = alloc(ctx, count, sizeof(int))))
            return rc;
        ZL_CUDA(ctx, cudaMemsetAsync(mark.ptr, 0, (size_t)cells * 4, ctx->stream));
        const int K = ctx->dims == 3 ? v.width * v.width * v.width : v.width * v.width;
        const unsigned blocks = (unsigned)(((long long)n * K + 127) / 128);
        if (ctx->dims == 2)
            ib_mark_kernel<2><<<blocks, 128, 0, ctx->stream>>>(L.geo, L.map, v, (uint32_t*)mark.ptr,
                                                              (int*)ctx->scratch_flag.ptr);
        else
            ib_mark_kernel<3><<<blocks, 128, 0, ctx->stream>>>(L.geo, L.map, v, (uint32_t*)mark.ptr,
                                                              (int*)ctx->scratch_flag.ptr);
        ZL_CUDA(ctx, cudaGetLastError());
        int bad = 0;
        if ((rc = read_flag(ctx, &bad))) return rc;
        if (bad) {
            if ((rc = release(nullptr))) return rc;
            return fail(ctx, ZL_ETOPOLOGY, "level %d: an immersed-boundary stencil node is not on the level", level);
        }
        if ((rc = release(mark.ptr))) return rc;
        size_t tmp_bytes = 0;
        ZL_CUDA(ctx, select_marked((const uint32_t*)mark.ptr, (int)cells, (int*)sel.ptr, (int*)count.ptr, nullptr,
                                   &tmp_bytes, ctx->stream));
        if ((rc = alloc(ctx, tmp, std::max<size_t>(tmp_bytes, 1)))) return rc;
        ZL_CUDA(ctx, select_marked((const uint32_t*)mark.ptr, (int)cells, (int*)sel.ptr, (int*)count.ptr, tmp.ptr,
                                   &tmp_bytes, ctx->stream));
        int nodes = 0;
        ZL_CUDA(ctx, cudaMemcpyAsync(&nodes, count.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if ((rc = alloc(ctx, L.ib_nodes, (size_t)std::max(nodes, 1) * 4))) return rc;
        ZL_CUDA(ctx, cudaMemcpyAsync(L.ib_nodes.ptr, sel.ptr, (size_t)nodes * 4, cudaMemcpyDeviceToDevice, ctx->stream));
        // the stencils resolved once: every (vertex, stencil node) pair's cell and delta weight, and
        // each stencil node's pairs in vertex order (stable sort on the node's list index)
        const long long pairs = (long long)n * K;
        if (pairs >= 0x7fffffffll) return fail(ctx, ZL_ETOOLARGE, "level %d: too many vertex-node pairs", level);
        {
            DeviceBuffer node_of_cell, key, key_sorted, id, csr_pair, stmp;
            if ((rc = alloc(ctx, node_of_cell, (size_t)cells * 4)) || (rc = alloc(ctx, key, (size_t)pairs * 4)) ||
                (rc = alloc(ctx, key_sorted, (size_t)pairs * 4)) || (rc = alloc(ctx, id, (size_t)pairs * 4)) ||
                (rc = alloc(ctx, csr_pair, (size_t)pairs * 4)) ||
                (rc = alloc(ctx, L.ib_pair_cell, (size_t)pairs * 4)) || (rc = alloc(ctx, L.ib_pair_w, (size_t)pairs * 8)) ||
                (rc = alloc(ctx, L.ib_csr_vertex, (size_t)pairs * 4)) ||
                (rc = alloc(ctx, L.ib_csr_share, (size_t)pairs * 8)) ||
                (rc = alloc(ctx, L.ib_csr_start, (size_t)(nodes + 1) * 4)))
                return rc;
            ib_index_nodes_kernel<<<(nodes + 127) / 128, 128, 0, ctx->stream>>>((const int*)L.ib_nodes.ptr, nodes,
                                                                               (int*)node_of_cell.ptr);
            const unsigned pblocks = (unsigned)((pairs + 127) / 128);
            if (ctx->dims == 2)
                ib_pairs_kernel<2><<<pblocks, 128, 0, ctx->stream>>>(L.geo, L.map, v, (const int*)node_of_cell.ptr,
                                                                    (int*)L.ib_pair_cell.ptr, (double*)L.ib_pair_w.ptr,
                                                                    (int*)key.ptr, (int*)id.ptr);
            else
                ib_pairs_kernel<3><<<pblocks, 128, 0, ctx->stream>>>(L.geo, L.map, v, (const int*)node_of_cell.ptr,
                                                                    (int*)L.ib_pair_cell.ptr, (double*)L.ib_pair_w.ptr,
                                                                    (int*)key.ptr, (int*)id.ptr);
            ZL_CUDA(ctx, cudaGetLastError());
            int bits = 1;
            while ((1ll << bits) < (long long)nodes) ++bits;
            size_t sbytes = 0;
            ZL_CUDA(ctx, sort_pairs_by_key((const int*)key.ptr, (int*)key_sorted.ptr, (const int*)id.ptr,
                                           (int*)csr_pair.ptr, (int)pairs, bits, nullptr, &sbytes, ctx->stream));
            if ((rc = alloc(ctx, stmp, std::max<size_t>(sbytes, 1)))) return rc;
            ZL_CUDA(ctx, sort_pairs_by_key((const int*)key.ptr, (int*)key_sorted.ptr, (const int*)id.ptr,
                                           (int*)csr_pair.ptr, (int)pairs, bits, stmp.ptr, &sbytes, ctx->stream));
            ib_csr_start_kernel<<<(unsigned)((pairs + 1 + 127) / 128), 128, 0, ctx->stream>>>(
                (const int*)key_sorted.ptr, pairs, (int*)L.ib_csr_start.ptr, nodes);
            if (ctx->dims == 2)
                ib_csr_fill_kernel<2><<<pblocks, 128, 0, ctx->stream>>>(v, L.params.dt, (const int*)csr_pair.ptr,
                                                                       (const double*)L.ib_pair_w.ptr, pairs,
                                                                       (int*)L.ib_csr_vertex.ptr, (double*)L.ib_csr_share.ptr);
            else
                ib_csr_fill_kernel<3><<<pblocks, 128, 0, ctx->stream>>>(v, L.params.dt, (const int*)csr_pair.ptr,
                                                                       (const double*)L.ib_pair_w.ptr, pairs,
                                                                       (int*)L.ib_csr_vertex.ptr, (double*)L.ib_csr_share.ptr);
            ZL_CUDA(ctx, cudaGetLastError());
            ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        }
        // the step reads node forces only where kInfoForce is set (forces elsewhere stay 0); the
        // bit is never cleared, released nodes keep it with a zero force
        if (L.info.ptr && nodes > 0) {
            or_bits_kernel<<<(nodes + 127) / 128, 128, 0, ctx->stream>>>((uint32_t*)L.info.ptr, (const int*)L.ib_nodes.ptr,
                                                                          nodes, kInfoForce);
            ZL_CUDA(ctx, cudaGetLastError());
        }
        ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        L.n_ib_nodes = nodes;
    }
    guard.done = true;
    return ZL_OK;
}

int zl_ib_set_delta(zl_ctx* ctx, int level, int width) {
    int rc = check_level(ctx, level, false);
    if (rc) return rc;
    if (width != ZL_IB_DELTA_4 && width != ZL_IB_DELTA_3) return fail(ctx, ZL_EINVAL, "stencil width %d", width);
    // the level's stencil-node list (and the cells that read node forces) follow the width
    if (ctx->levels[level].n_vertices > 0 && ctx->levels[level].ib_width != width)
        return fail(ctx, ZL_ESTATE, "level %d: set the delta kernel before the vertices", level);
    ctx->levels[level].ib_width = width;
    ++ctx->generation;
    return ZL_OK;
}

int zl_ib_get_forces(zl_ctx* ctx, int level, double* vertex_forces, double* total) {
    int rc = check_level(ctx, level, true);
    if (rc) return rc;
    Level& L = ctx->levels[level];
    if (L.n_vertices <= 0) return fail(ctx, ZL_ESTATE, "level %d has no immersed-boundary vertices", level);
    if (vertex_forces)
        ZL_CUDA(ctx, cudaMemcpyAsync(vertex_forces, L.ib_force.ptr, (size_t)L.n_vertices * 3 * 8,
                                     cudaMemcpyDeviceToHost, ctx->stream));
    if (total) {
        IbVertices v = ib_view(ctx, L, level);
        const double dx0 = ctx->cfg.dx > 0. ? ctx->cfg.dx : 1.;
        const double scale = ctx->dims == 3 ? 1. / dx0 / dx0 : 1. / dx0;
        ib_total_kernel<<<1, 32, 0, ctx->stream>>>(v, scale, (double*)L.ib_total.ptr);
        ZL_CUDA(ctx, cudaGetLastError());
        ZL_CUDA(ctx, cudaMemcpyAsync(total, L.ib_total.ptr, 3 * 8, cudaMemcpyDeviceToHost, ctx->stream));
    }
    ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return ZL_OK;
}

int zl_synchronize(zl_ctx* ctx) {
    if (!ctx) return ZL_EINVAL;
    ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->closure_err.ptr) {
        int e = 0;
        ZL_CUDA(ctx, cudaMemcpy(&e, ctx->closure_err.ptr, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) return fail(ctx, ZL_ETIMEOUT, "a tensor-core wait of the learned closure step timed out");
    }
    return ZL_OK;
}

int zl_get_stream(const zl_ctx* ctx, void** stream) {
    if (!ctx || !stream) return ZL_EINVAL;
    *stream = (void*)ctx->stream;
    return ZL_OK;
}

int zl_set_stream(zl_ctx* ctx, void* stream) {
    if (!ctx) return ZL_EINVAL;
    ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return ZL_OK;
}

int zl_last_error(const zl_ctx* ctx, char* buf, size_t n) {
    if (!ctx || !buf || n == 0) return ZL_EINVAL;
    std::snprintf(buf, n, "%s", ctx->last_error.c_str());
    return ZL_OK;
}

int zl_level_info(const zl_ctx* ctx, int level, int64_t* nodes, int32_t* extent, int64_t* pop_bytes) {
    if (!ctx || level < 0 || level >= ZL_MAX_LEVELS) return ZL_EINVAL;
    const Level& L = ctx->levels[level];
    if (nodes) *nodes = L.active ? L.nodes : 0;
    if (extent)
        for (int a = 0; a < 3; ++a) extent[a] = L.active ? L.geo.n[a] : 0;
    if (pop_bytes) *pop_bytes = L.active ? (int64_t)L.f.bytes : 0;
    return ZL_OK;
}

int zl_morton_neighbors(int dims, const uint64_t* codes, int64_t n, uint64_t* out) {
    if ((dims != 2 && dims != 3) || n < 0 || (n > 0 && (!codes || !out))) return ZL_EINVAL;
    if (n == 0) return ZL_OK;
    uint64_t *dc = nullptr, *dout = nullptr;
    if (cudaMalloc(&dc, n * 8) != cudaSuccess) return ZL_EDEVICE;
    if (cudaMalloc(&dout, n * 2 * dims * 8) != cudaSuccess) {
        cudaFree(dc);
        return ZL_EDEVICE;
    }
    int rc = ZL_OK;
    if (cudaMemcpy(dc, codes, n * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        launch_morton_neighbors(dc, n, dims, dout, 0) != cudaSuccess ||
        cudaMemcpy(out, dout, n * 2 * dims * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = ZL_EDEVICE;
    cudaFree(dc);
    cudaFree(dout);
    return rc;
}

int zl_upstream_index(int lattice, const uint64_t* codes, int64_t n, int64_t* out) {
    if ((lattice != ZL_D2Q9 && lattice != ZL_D3Q19) || n < 0 || (n > 0 && (!codes || !out))) return ZL_EINVAL;
    if (n == 0) return ZL_OK;
    const int dims = lattice == ZL_D2Q9 ? 2 : 3, q = dims == 2 ? 9 : 19;
    // sort codes on the host side of the call (set-up path), resolve on the device
    std::vector<std::pair<uint64_t, long long>> order(n);
    for (int64_t i = 0; i < n; ++i) order[i] = {codes[i], (long long)i};
    std::sort(order.begin(), order.end());
    std::vector<uint64_t> sorted(n);
    std::vector<long long> pos(n);
    for (int64_t i = 0; i < n; ++i) {
        sorted[i] = order[i].first;
        pos[i] = order[i].second;
    }
    uint64_t* ds = nullptr;
    long long *dp = nullptr, *dout = nullptr;
    int rc = ZL_OK;
    if (cudaMalloc(&ds, n * 8) != cudaSuccess || cudaMalloc(&dp, n * 8) != cudaSuccess ||
        cudaMalloc(&dout, (size_t)n * q * 8) != cudaSuccess) {
        rc = ZL_EDEVICE;
    } else if (cudaMemcpy(ds, sorted.data(), n * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(dp, pos.data(), n * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
               launch_upstream_index(dims, ds, dp, n, dout, 0) != cudaSuccess ||
               cudaMemcpy(out, dout, (size_t)n * q * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
        rc = ZL_EDEVICE;
    }
    if (ds) cudaFree(ds);
    if (dp) cudaFree(dp);
    if (dout) cudaFree(dout);
    return rc;
}

int zl_mrt_matrix(int lattice, double tau, double* out) {
    if ((lattice != ZL_D2Q9 && lattice != ZL_D3Q19) || !out || !(tau > 0.)) return ZL_EINVAL;
    host_mrt_matrix(lattice == ZL_D2Q9 ? 2 : 3, 1. / tau, false, out);
    return ZL_OK;
}

}  // extern "C"

// A full-box D3Q19 level (the dense device I/O and closure kernels); the closure kernels need
// FP32 / FP16 / BF16 storage, the dense equilibrium and macro I/O take FP64 as well.
static int check_box_level(zl_ctx* ctx, int level, bool any_storage = false) {
    int rc = check_level(ctx, level, true);
    if (rc) return rc;
    const Level& L = ctx->levels[level];
    if (ctx->dims != 3) return fail(ctx, ZL_EINVAL, "dense level I/O and the closure need D3Q19");
    if (!any_storage && ctx->cfg.storage == ZL_STORAGE_F64)
        return fail(ctx, ZL_EINVAL, "the closure kernels need FP32/FP16/BF16 storage");
    if (L.nodes != (long long)L.geo.n[0] * L.geo.n[1] * L.geo.n[2])
        return fail(ctx, ZL_EINVAL, "level %d is not a full box", level);
    return ZL_OK;
}

extern "C" {

int zl_set_equilibrium_dense(zl_ctx* ctx, int level, const float* rho_device, const float* u_device) {
    int rc = check_box_level(ctx, level, true);
    if (rc) return rc;
    if (!rho_device || !u_device) return fail(ctx, ZL_EINVAL, "null field");
    Level& L = ctx->levels[level];
    ZL_CUDA(ctx, closure_box_op(kBoxSetEq, ctx->cfg.storage, L.f.ptr, L.geo, L.params, L.even_layout, rho_device,
                                const_cast<float*>(u_device), nullptr, 0, nullptr, ctx->stream));
    return ZL_OK;
}

int zl_get_macros_dense(zl_ctx* ctx, int level, float* rho_device, float* u_device) {
    int rc = check_box_level(ctx, level, true);
    if (rc) return rc;
    if (!rho_device || !u_device) return fail(ctx, ZL_EINVAL, "null field");
    Level& L = ctx->levels[level];
    ZL_CUDA(ctx, closure_box_op(kBoxGetMacros, ctx->cfg.storage, L.f.ptr, L.geo, L.params, L.even_layout, nullptr,
                                rho_device, u_device, 0, nullptr, ctx->stream));
    return ZL_OK;
}

int zl_closure_features(zl_ctx* ctx, int level, float* x_device) {
    int rc = check_box_level(ctx, level);
    if (rc) return rc;
    if (!x_device) return fail(ctx, ZL_EINVAL, "null output");
    Level& L = ctx->levels[level];
    ZL_CUDA(ctx, closure_box_op(kBoxFeatures, ctx->cfg.storage, L.f.ptr, L.geo, L.params, L.even_layout, nullptr,
                                x_device, nullptr, 0, nullptr, ctx->stream));
    return ZL_OK;
}

int zl_filter_level(zl_ctx* ctx, int level, int factor, float* out_device) {
    int rc = check_box_level(ctx, level);
    if (rc) return rc;
    Level& L = ctx->levels[level];
    if (!out_device || factor < 1) return fail(ctx, ZL_EINVAL, "bad filter arguments");
    int nc[3];
    for (int a = 0; a < 3; ++a) {
        if (L.geo.n[a] % factor) return fail(ctx, ZL_EINVAL, "axis %d: %d nodes not a multiple of %d", a, L.geo.n[a], factor);
        nc[a] = L.geo.n[a] / factor;
    }
    ZL_CUDA(ctx, closure_box_op(kBoxFilter, ctx->cfg.storage, L.f.ptr, L.geo, L.params, L.even_layout, nullptr,
                                out_device, nullptr, factor, nc, ctx->stream));
    return ZL_OK;
}

int zl_set_closure_interval(zl_ctx* ctx, int every) {
    if (!ctx || every < 1) return ZL_EINVAL;
    ctx->closure_every = every;
    ++ctx->generation;
    return ZL_OK;
}

int zl_set_closure(zl_ctx* ctx, const zl_mlp* net) {
    if (!ctx) return ZL_EINVAL;
    ZL_CUDA(ctx, cudaSetDevice(ctx->cfg.device));
    ++ctx->generation;
    if (!net) {
        ctx->closure_net.release();
        return ZL_OK;
    }
    int rc = ctx->closure_net.ptr ? ZL_OK : alloc(ctx, ctx->closure_net, sizeof(zl_mlp));
    if (rc) return rc;
    if (!ctx->closure_err.ptr) {
        if ((rc = alloc(ctx, ctx->closure_err, sizeof(int)))) return rc;
        ZL_CUDA(ctx, cudaMemsetAsync(ctx->closure_err.ptr, 0, sizeof(int), ctx->stream));
    }
    ZL_CUDA(ctx, cudaMemcpyAsync(ctx->closure_net.ptr, net, sizeof(zl_mlp), cudaMemcpyHostToDevice, ctx->stream));
    ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return ZL_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- checkpoint node records
// Cell of a code on a level (the code must belong to the level; periodic duplicates wrap).
static long long cell_of_level_code(const Level& L, int dims, uint64_t code) {
    uint32_t idx[3];
    zl::morton_decode(code, dims, idx);
    long long b[3] = {0, 0, 0};
    for (int a = 0; a < dims; ++a) {
        long long v = (long long)idx[a] - L.map.lo[a];
        if (L.map.periodic[a] && v == L.map.n[a]) v = 0;
        if (v < 0 || v >= L.map.n[a]) return -1;
        b[a] = v + L.geo.g[a];
    }
    return b[0] + (long long)L.geo.a[0] * (b[1] + (long long)L.geo.a[1] * b[2]);
}

extern "C" {

int zl_write_checkpoint_nodes(zl_ctx* ctx, const char* path, const uint64_t* const* codes,
                              const int32_t* const* flags, const int64_t* n) {
    if (!ctx || !path || !codes || !flags || !n) return ZL_EINVAL;
    const int dims = ctx->dims, q = ctx->q, levels = ctx->cfg.max_level + 1;
    const int n_forces = ctx->cfg.forcing ? dims : 0;
    struct Key {
        uint64_t cell;
        int level;
        long long local, index;
    };
    std::vector<Key> keys;
    std::vector<std::vector<double>> f(levels), force(levels);
    for (int l = 0; l < levels; ++l) {
        int rc = check_level(ctx, l, true);
        if (rc) return rc;
        if (n[l] < 0 || (n[l] > 0 && (!codes[l] || !flags[l]))) return fail(ctx, ZL_EINVAL, "level %d: bad node list", l);
        f[l].resize((size_t)n[l] * q);
        if (n[l] > 0 && (rc = zl_get_populations(ctx, l, codes[l], f[l].data(), n[l]))) return rc;
        const Level& L = ctx->levels[l];
        if (n_forces) {
            // the node forces of the last forcing pass (GridNodeLbm::force_)
            const long long cells = (long long)L.geo.a[0] * L.geo.a[1] * L.geo.a[2];
            std::vector<double> all((size_t)cells * 3);
            ZL_CUDA(ctx, cudaMemcpy(all.data(), L.force.ptr, all.size() * sizeof(double), cudaMemcpyDeviceToHost));
            force[l].resize((size_t)n[l] * n_forces);
            for (int64_t i = 0; i < n[l]; ++i) {
                const long long c = cell_of_level_code(L, dims, codes[l][i]);
                if (c < 0) return fail(ctx, ZL_ETOPOLOGY, "level %d: code not on the level", l);
                for (int a = 0; a < n_forces; ++a) force[l][(size_t)i * n_forces + a] = all[(size_t)c * 3 + a];
            }
        }
        // background cell (SFBitsetToNLowerLevel), then x-y-z order inside the cell
        // (SFBitsetHigherLevelInACell, sfbitset_aux.cpp:140-156, :1958-1985)
        const uint64_t side = 1ull << l;
        for (int64_t i = 0; i < n[l]; ++i) {
            uint32_t idx[3];
            zl::morton_decode(codes[l][i], dims, idx);
            long long local = 0;
            for (int a = dims - 1; a >= 0; --a) local = local * (long long)side + (long long)(idx[a] & (side - 1));
            keys.push_back({codes[l][i] >> (dims * l), l, local, i});
        }
    }
    std::sort(keys.begin(), keys.end(), [](const Key& a, const Key& b) {
        if (a.cell != b.cell) return a.cell < b.cell;
        if (a.level != b.level) return a.level < b.level;
        return a.local < b.local;
    });
    const int32_t data_size = 4 + 8 * q + 8 * n_forces;
    const size_t node_size = 8 + 4 + (size_t)data_size;
    if (keys.size() > 0xffffffffull) return fail(ctx, ZL_ETOOLARGE, "more than 2^32 nodes");
    std::vector<char> buf(8 + keys.size() * node_size);
    const uint32_t total = (uint32_t)keys.size();
    std::memcpy(buf.data(), &total, 4);
    std::memcpy(buf.data() + 4, &data_size, 4);
    char* p = buf.data() + 8;
    for (const Key& k : keys) {
        const int32_t lv = k.level;
        std::memcpy(p, &codes[lv][k.index], 8);
        std::memcpy(p + 8, &lv, 4);
        std::memcpy(p + 12, &flags[lv][k.index], 4);
        std::memcpy(p + 16, &f[lv][(size_t)k.index * q], (size_t)q * 8);
        if (n_forces) std::memcpy(p + 16 + q * 8, &force[lv][(size_t)k.index * n_forces], (size_t)n_forces * 8);
        p += node_size;
    }
    FILE* fh = std::fopen(path, "wb");
    if (!fh) return fail(ctx, ZL_EINVAL, "cannot open %s", path);
    const size_t w = std::fwrite(buf.data(), 1, buf.size(), fh);
    std::fclose(fh);
    if (w != buf.size()) return fail(ctx, ZL_EINVAL, "short write to %s", path);
    return ZL_OK;
}

int zl_read_checkpoint_nodes(zl_ctx* ctx, const char* path) {
    if (!ctx || !path) return ZL_EINVAL;
    const int q = ctx->q, levels = ctx->cfg.max_level + 1;
    FILE* fh = std::fopen(path, "rb");
    if (!fh) return fail(ctx, ZL_EINVAL, "cannot open %s", path);
    uint32_t total = 0;
    int32_t data_size = 0;
    if (std::fread(&total, 4, 1, fh) != 1 || std::fread(&data_size, 4, 1, fh) != 1) {
        std::fclose(fh);
        return fail(ctx, ZL_EINVAL, "%s: no checkpoint header", path);
    }
    const int extra = data_size - 4 - 8 * q;
    if (extra < 0 || extra % 8) {
        std::fclose(fh);
        return fail(ctx, ZL_EINVAL, "%s: node data of %d bytes does not hold %d populations", path, data_size, q);
    }
    const size_t node_size = 12 + (size_t)data_size;
    std::vector<char> buf((size_t)total * node_size);
    const size_t got = buf.empty() ? 0 : std::fread(buf.data(), node_size, total, fh);
    std::fclose(fh);
    if (got != total) return fail(ctx, ZL_EINVAL, "%s: %zu of %u node records", path, got, total);
    std::vector<std::vector<uint64_t>> codes(levels);
    std::vector<std::vector<double>> f(levels);
    for (uint32_t i = 0; i < total; ++i) {
        const char* p = buf.data() + (size_t)i * node_size;
        uint64_t code;
        int32_t lv;
        std::memcpy(&code, p, 8);
        std::memcpy(&lv, p + 8, 4);
        if (lv < 0 || lv >= levels) return fail(ctx, ZL_ETOPOLOGY, "%s: record of level %d", path, lv);
        codes[lv].push_back(code);
        const size_t o = f[lv].size();
        f[lv].resize(o + q);
        std::memcpy(&f[lv][o], p + 16, (size_t)q * 8);
    }
    for (int l = 0; l < levels; ++l) {
        if (codes[l].empty()) continue;
        const int rc = zl_set_populations(ctx, l, codes[l].data(), f[l].data(), (int64_t)codes[l].size());
        if (rc) return rc;
    }
    return ZL_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- VTK XML field output
namespace {

// One binary DataArray body: base64 text of the device payload, built on the device.
int vtu_binary_array(zl_ctx* ctx, FILE* fp, const void* dpayload, size_t nbytes) {
    if (nbytes > 0xffffffffull) return fail(ctx, ZL_ETOOLARGE, "a VTK array above 4 GiB (UInt32 header)");
    const unsigned long long nchars = base64_chars(nbytes);
    DeviceBuffer dtext;
    int rc = alloc(ctx, dtext, (size_t)nchars);
    if (rc) return rc;
    ZL_CUDA(ctx, base64_encode(dpayload, nbytes, (char*)dtext.ptr, ctx->stream));
    std::vector<char> text(nchars);
    ZL_CUDA(ctx, cudaMemcpyAsync(text.data(), dtext.ptr, nchars, cudaMemcpyDeviceToHost, ctx->stream));
    ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (std::fwrite(text.data(), 1, nchars, fp) != nchars || std::fputc('\n', fp) == EOF)
        return fail(ctx, ZL_EINVAL, "short write of a VTK file");
    return ZL_OK;
}

template <class T>
int vtu_fetch(zl_ctx* ctx, std::vector<T>& host, const void* dptr, size_t count) {
    host.resize(count);
    if (count) ZL_CUDA(ctx, cudaMemcpyAsync(host.data(), dptr, count * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return ZL_OK;
}

// SFBitsetComputeCoordinate (morton_aux.cpp:86-101, :310-333), for the ASCII form
double vtu_coordinate(uint64_t code, int dims, int axis, int level, double space, double origin) {
    const double gs = space / (double)(1ull << level);
    double c = origin;
    for (int b = 0; b < 64 / dims; ++b)
        if ((code >> (dims * b + axis)) & 1ull) c += gs * (double)(1ull << b);
    return c;
}

int vtu_level(zl_ctx* ctx, const std::string& path, int level, bool binary, const double* space, const double* origin,
              uint32_t ghost_mask, const uint64_t* codes, const int32_t* flags, int64_t n) {
    const int dims = ctx->dims;
    const int corners = dims == 2 ? 4 : 8;
    Level& L = ctx->levels[level];
    if (n < 0 || n > 0x7fffffffll || (n > 0 && (!codes || !flags)))
        return fail(ctx, ZL_EINVAL, "level %d: bad point list", level);
    DeviceBuffer dcodes, dflags, dmac, dflag16, dghost, drho32, du32, dxyz, dtable, dcell, dfirst, dscan, dconn,
        doffs, dtypes;
    int rc;
    if ((rc = upload_codes(ctx, codes, n, dcodes))) return rc;
    if ((rc = alloc(ctx, dflags, (size_t)std::max<int64_t>(n, 1) * 4))) return rc;
    if (n) ZL_CUDA(ctx, cudaMemcpyAsync(dflags.ptr, flags, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
    // density and velocity recomputed from the current populations (the values the reference's
    // "velocity" output variable computes, lbm_grid_interface.cpp:645-652)
    if ((rc = alloc(ctx, dmac, (size_t)std::max<int64_t>(n, 1) * (dims + 1) * sizeof(double)))) return rc;
    double* drho = (double*)dmac.ptr;
    double* du = drho + n;
    if (n) {
        if ((rc = reset_flag(ctx))) return rc;
        ZL_CUDA(ctx, ctx->ops->gather(dims, L.f.ptr, L.geo, L.params, L.map, L.even_layout,
                                      (const uint64_t*)dcodes.ptr, nullptr, drho, du, n, (int*)ctx->scratch_flag.ptr,
                                      ctx->stream));
        int bad = 0;
        if ((rc = read_flag(ctx, &bad))) return rc;
        if (bad) return fail(ctx, ZL_ETOPOLOGY, "level %d: a point code is not part of the level", level);
    }
    // index box of the points -> point table
    VtuLevel a{};
    a.codes = (const uint64_t*)dcodes.ptr;
    a.flags = (const int32_t*)dflags.ptr;
    a.n = n;
    a.dims = dims;
    a.level = level;
    for (int d = 0; d < 3; ++d) {
        a.space[d] = space[d];
        a.origin[d] = origin[d];
        a.lo[d] = 0;
        a.ext[d] = 1;
    }
    a.ghost_mask = ghost_mask;
    long long table_cells = 1;
    if (n) {
        DeviceBuffer dmm;
        if ((rc = alloc(ctx, dmm, 6 * sizeof(int)))) return rc;
        int mm[6] = {INT32_MAX, INT32_MAX, INT32_MAX, 0, 0, 0};
        ZL_CUDA(ctx, cudaMemcpyAsync(dmm.ptr, mm, sizeof(mm), cudaMemcpyHostToDevice, ctx->stream));
        ZL_CUDA(ctx, launch_decode_minmax(a.codes, n, dims, (int*)dmm.ptr, ctx->stream));
        ZL_CUDA(ctx, cudaMemcpyAsync(mm, dmm.ptr, sizeof(mm), cudaMemcpyDeviceToHost, ctx->stream));
        ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        for (int d = 0; d < dims; ++d) {
            a.lo[d] = mm[d];
            a.ext[d] = (long long)mm[3 + d] - mm[d] + 1;
            table_cells *= a.ext[d];
        }
    }
    const size_t nn = (size_t)std::max<int64_t>(n, 1);
    if ((rc = alloc(ctx, dtable, (size_t)table_cells * 4))) return rc;
    ZL_CUDA(ctx, cudaMemsetAsync(dtable.ptr, 0xff, (size_t)table_cells * 4, ctx->stream));
    if ((rc = alloc(ctx, dflag16, nn * 2)) || (rc = alloc(ctx, dghost, nn)) || (rc = alloc(ctx, drho32, nn * 4)) ||
        (rc = alloc(ctx, du32, nn * dims * 4)) || (rc = alloc(ctx, dxyz, nn * 12)) || (rc = alloc(ctx, dcell, nn * 4)) ||
        (rc = alloc(ctx, dfirst, nn * 4)))
        return rc;
    ZL_CUDA(ctx, vtu_points(a, drho, du, (uint16_t*)dflag16.ptr, (uint8_t*)dghost.ptr, (float*)drho32.ptr,
                            (float*)du32.ptr, (float*)dxyz.ptr, (int32_t*)dtable.ptr, ctx->stream));
    const size_t scan_bytes = std::max<size_t>(vtu_scan_bytes(n), 1);
    if ((rc = alloc(ctx, dscan, scan_bytes))) return rc;
    ZL_CUDA(ctx, vtu_cells(a, (const int32_t*)dtable.ptr, (uint32_t*)dcell.ptr, (uint32_t*)dfirst.ptr, dscan.ptr,
                           scan_bytes, ctx->stream));
    long long cells = 0;
    if (n) {
        uint32_t last[2];
        ZL_CUDA(ctx, cudaMemcpyAsync(&last[0], (uint32_t*)dfirst.ptr + (n - 1), 4, cudaMemcpyDeviceToHost, ctx->stream));
        ZL_CUDA(ctx, cudaMemcpyAsync(&last[1], (uint32_t*)dcell.ptr + (n - 1), 4, cudaMemcpyDeviceToHost, ctx->stream));
        ZL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        cells = (long long)last[0] + last[1];
    }
    const size_t nc = (size_t)std::max<long long>(cells, 1);
    if ((rc = alloc(ctx, dconn, nc * corners * 8)) || (rc = alloc(ctx, doffs, nc * 8)) || (rc = alloc(ctx, dtypes, nc)))
        return rc;
    ZL_CUDA(ctx, vtu_connect(a, (const int32_t*)dtable.ptr, (const uint32_t*)dcell.ptr, (const uint32_t*)dfirst.ptr,
                             (uint64_t*)dconn.ptr, ctx->stream));
    ZL_CUDA(ctx, vtu_offsets(cells, dims, (uint64_t*)doffs.ptr, (uint8_t*)dtypes.ptr, ctx->stream));

    FILE* fp = std::fopen(path.c_str(), "w");
    if (!fp) return fail(ctx, ZL_EINVAL, "cannot open %s", path.c_str());
    struct Closer {
        FILE* f;
        ~Closer() { std::fclose(f); }
    } closer{fp};
    const char* fmt = binary ? "binary" : "ascii";
    std::fprintf(fp, "<?xml version=\"1.0\"?>\n");
    std::fprintf(fp, "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
    std::fprintf(fp, " <UnstructuredGrid>\n");
    std::fprintf(fp, "  <Piece NumberOfPoints=\"%lld\" NumberOfCells=\"%lld\">\n", (long long)n, cells);
    std::fprintf(fp, "    <PointData>\n");
    // host copies for the ASCII form (the reference prints the FP64 values with %f)
    std::vector<double> hmac;
    std::vector<uint64_t> hconn;
    if (!binary) {
        if ((rc = vtu_fetch(ctx, hmac, dmac.ptr, (size_t)n * (dims + 1)))) return rc;
        if ((rc = vtu_fetch(ctx, hconn, dconn.ptr, (size_t)cells * corners))) return rc;
    }
    std::fprintf(fp, "      <DataArray NumberOfComponents=\"1\" type=\"UInt16\" Name=\"flag_status\" format=\"%s\">\n",
                 fmt);
    if (binary) {
        if ((rc = vtu_binary_array(ctx, fp, dflag16.ptr, (size_t)n * 2))) return rc;
    } else {
        for (int64_t i = 0; i < n; ++i) std::fprintf(fp, "       %hu\n", (unsigned short)flags[i]);
    }
    std::fprintf(fp, "      </DataArray>\n");
    std::fprintf(fp, "      <DataArray type=\"UInt8\" Name=\"vtkGhostType\" format=\"%s\">\n", fmt);
    if (binary) {
        if ((rc = vtu_binary_array(ctx, fp, dghost.ptr, (size_t)n))) return rc;
    } else {
        for (int64_t i = 0; i < n; ++i) std::fprintf(fp, "   %u\n", (flags[i] & (int32_t)ghost_mask) != 0 ? 1u : 0u);
    }
    std::fprintf(fp, "      </DataArray>\n");
    // output variables in std::set order: "rho", "velocity"
    std::fprintf(fp, "      <DataArray NumberOfComponents=\"1\" type=\"Float32\" Name=\"rho\" format=\"%s\">\n", fmt);
    if (binary) {
        if ((rc = vtu_binary_array(ctx, fp, drho32.ptr, (size_t)n * 4))) return rc;
    } else {
        for (int64_t i = 0; i < n; ++i) std::fprintf(fp, "       %f\n", hmac[i]);
    }
    std::fprintf(fp, "      </DataArray>\n");
    std::fprintf(fp, "      <DataArray NumberOfComponents=\"%d\" type=\"Float32\" Name=\"velocity\" format=\"%s\">\n",
                 dims, fmt);
    if (binary) {
        if ((rc = vtu_binary_array(ctx, fp, du32.ptr, (size_t)n * dims * 4))) return rc;
    } else {
        for (int64_t i = 0; i < n; ++i) {
            for (int d = 0; d < dims; ++d) std::fprintf(fp, "       %f", hmac[n + i * dims + d]);
            std::fprintf(fp, "\n");
        }
    }
    std::fprintf(fp, "      </DataArray>\n");
    std::fprintf(fp, "    </PointData>\n");
    std::fprintf(fp, "   <Points>\n");
    std::fprintf(fp, "    <DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"%s\">\n", fmt);
    if (binary) {
        if ((rc = vtu_binary_array(ctx, fp, dxyz.ptr, (size_t)n * 12))) return rc;
    } else {
        for (int64_t i = 0; i < n; ++i) {
            double c[3] = {0., 0., 0.};
            for (int d = 0; d < dims; ++d) c[d] = vtu_coordinate(codes[i], dims, d, level, space[d], origin[d]);
            std::fprintf(fp, "   %f %f %f\n", c[0], c[1], c[2]);
        }
    }
    std::fprintf(fp, "    </DataArray>\n");
    std::fprintf(fp, "   </Points>\n");
    std::fprintf(fp, "   <Cells>\n");
    std::fprintf(fp, "    <DataArray type=\"UInt64\" Name=\"connectivity\" format=\"%s\">\n", fmt);
    if (binary) {
        if ((rc = vtu_binary_array(ctx, fp, dconn.ptr, (size_t)cells * corners * 8))) return rc;
    } else {
        for (long long c = 0; c < cells; ++c) {
            std::fprintf(fp, "  ");
            for (int k = 0; k < corners; ++k) std::fprintf(fp, " %llu", (unsigned long long)hconn[c * corners + k]);
            std::fprintf(fp, "\n");
        }
    }
    std::fprintf(fp, "    </DataArray>\n");
    std::fprintf(fp, "    <DataArray type=\"UInt64\" Name=\"offsets\" format=\"%s\">\n", fmt);
    if (binary) {
        if ((rc = vtu_binary_array(ctx, fp, doffs.ptr, (size_t)cells * 8))) return rc;
    } else {
        for (long long c = 1; c <= cells; ++c) std::fprintf(fp, "   %llu\n", (unsigned long long)(c * corners));
    }
    std::fprintf(fp, "    </DataArray>\n");
    std::fprintf(fp, "    <DataArray type=\"UInt8\" Name=\"types\" format=\"%s\">\n", fmt);
    if (binary) {
        if ((rc = vtu_binary_array(ctx, fp, dtypes.ptr, (size_t)cells))) return rc;
    } else {
        for (long long c = 0; c < cells; ++c) std::fprintf(fp, "   %u\n", dims == 2 ? 8u : 11u);
    }
    std::fprintf(fp, "    </DataArray>\n");
    std::fprintf(fp, "   </Cells>\n");
    std::fprintf(fp, "  </Piece>\n");
    std::fprintf(fp, " </UnstructuredGrid>\n");
    std::fprintf(fp, "</VTKFile>");
    if (std::ferror(fp)) return fail(ctx, ZL_EINVAL, "write error on %s", path.c_str());
    return ZL_OK;
}

}  // namespace

int zl_write_vtu(zl_ctx* ctx, const char* prefix, int binary, const double* space, const double* origin,
                 uint32_t ghost_mask, const uint64_t* const* codes, const int32_t* const* flags, const int64_t* n) {
    if (!ctx || !prefix || !space || !origin || !codes || !flags || !n) return ZL_EINVAL;
    const int levels = ctx->cfg.max_level + 1;
    ZL_CUDA(ctx, cudaSetDevice(ctx->cfg.device));
    for (int l = 0; l < levels; ++l) {
        const int rc = check_level(ctx, l, true);
        if (rc) return rc;
    }
    const std::string folder = std::string(prefix) + "_data";
    std::error_code ec;
    std::filesystem::create_directories(folder, ec);
    if (ec) return fail(ctx, ZL_EINVAL, "cannot create %s", folder.c_str());
    for (int l = 0; l < levels; ++l) {
        const int rc = vtu_level(ctx, folder + "/rank_0_grid_level_" + std::to_string(l) + ".vtu", l, binary != 0,
                                 space, origin, ghost_mask, codes[l], flags[l], n[l]);
        if (rc) return rc;
    }
    // WritePvtu (vtk_writer_manager.cpp:296-372)
    const std::string pv = folder + "/rank_0_.pvtu";
    FILE* fp = std::fopen(pv.c_str(), "w");
    if (!fp) return fail(ctx, ZL_EINVAL, "cannot open %s", pv.c_str());
    const char* fmt = binary ? "binary" : "ascii";
    std::fprintf(fp, "<?xml version=\"1.0\"?>\n");
    std::fprintf(fp, "<VTKFile type=\"PUnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
    std::fprintf(fp, " <PUnstructuredGrid>\n");
    std::fprintf(fp, "    <PPointData>\n");
    std::fprintf(fp, "      <PDataArray NumberOfComponents=\"1\" type=\"UInt16\" Name=\"flag_status\" format=\"%s\">\n",
                 fmt);
    std::fprintf(fp, "      </PDataArray>\n");
    std::fprintf(fp, "      <PDataArray NumberOfComponents=\"1\" type=\"Float32\" Name=\"rho\" format=\"%s\">\n", fmt);
    std::fprintf(fp, "      </PDataArray>\n");
    std::fprintf(fp, "      <PDataArray NumberOfComponents=\"%d\" type=\"Float32\" Name=\"velocity\" format=\"%s\">\n",
                 ctx->dims, fmt);
    std::fprintf(fp, "      </PDataArray>\n");
    std::fprintf(fp, "      <PDataArray type=\"UInt8\" Name=\"vtkGhostType\" format=\"%s\">\n", fmt);
    std::fprintf(fp, "      </PDataArray>\n");
    std::fprintf(fp, "    </PPointData>\n");
    std::fprintf(fp, "   <PPoints>\n");
    std::fprintf(fp, "    <PDataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"%s\">\n", fmt);
    std::fprintf(fp, "    </PDataArray>\n");
    std::fprintf(fp, "   </PPoints>\n");
    std::fprintf(fp, "   <PCells>\n");
    std::fprintf(fp, "    <PDataArray type=\"UInt64\" Name=\"connectivity\" format=\"%s\">\n", fmt);
    std::fprintf(fp, "    </PDataArray>\n");
    std::fprintf(fp, "    <PDataArray type=\"UInt64\" Name=\"offsets\" format=\"%s\">\n", fmt);
    std::fprintf(fp, "    </PDataArray>\n");
    std::fprintf(fp, "    <PDataArray type=\"UInt8\" Name=\"types\" format=\"%s\">\n", fmt);
    std::fprintf(fp, "    </PDataArray>\n");
    std::fprintf(fp, "   </PCells>\n");
    for (int l = 0; l < levels; ++l) std::fprintf(fp, "    <Piece Source=\"rank_0_grid_level_%d.vtu\"/>\n", l);
    std::fprintf(fp, " </PUnstructuredGrid>\n");
    std::fprintf(fp, " </VTKFile>\n");
    const bool err = std::ferror(fp) != 0;
    std::fclose(fp);
    if (err) return fail(ctx, ZL_EINVAL, "write error on %s", pv.c_str());
    return ZL_OK;
}
