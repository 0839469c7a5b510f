// Device-side topology: Morton decode, axis-neighbour codes, upstream-node
// resolution and the per-level presence / boundary information.
//
// The neighbour arithmetic restates the reference's SFBitsetAux{2D,3D}::Find{X,Y,Z}{Neg,Pos}
// (amr_project/grid/morton_aux.hpp:65-297) on 64-bit integers: a Neg step on a zero axis
// field returns the input code unchanged, a Pos step carries through the other axes' bits.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include "topology.cuh"

namespace zl {

__global__ void decode_minmax_kernel(const uint64_t* __restrict__ codes, long long n, int dims,
                                     int* __restrict__ minmax) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t idx[3];
    morton_decode(codes[i], dims, idx);
    for (int a = 0; a < dims; ++a) {
        atomicMin(minmax + a, (int)idx[a]);
        atomicMax(minmax + 3 + a, (int)idx[a]);
    }
}

__global__ void mark_present_kernel(const uint64_t* __restrict__ codes, long long n, LevelMap m, LevelGeom geo,
                                    uint32_t* __restrict__ info, int* __restrict__ bad) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Coord c;
    if (!code_to_node(codes[i], m, c)) {
        atomicExch(bad, 1);
        return;
    }
    const long long cell = (long long)(c.x[0] + geo.g[0]) +
                           (long long)geo.a[0] * ((c.x[1] + geo.g[1]) + (long long)geo.a[1] * (c.x[2] + geo.g[2]));
    atomicOr(info + cell, kInfoPresent);
}

__global__ void count_present_kernel(const uint32_t* __restrict__ info, long long cells,
                                     unsigned long long* __restrict__ count) {
    unsigned long long local = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cells;
         i += (long long)gridDim.x * blockDim.x)
        local += (info[i] & kInfoPresent) ? 1ull : 0ull;
    for (int off = 16; off > 0; off >>= 1) local += __shfl_down_sync(0xffffffffu, local, off);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

// Missing-upstream bits and boundary-face bits of every present node.
template <class L>
// halo: faces whose ghost plane holds a neighbouring slab's slots (upstream nodes beyond such a
// face are missing only if their ghost cell is absent)
__global__ void node_info_kernel(LevelGeom geo, uint32_t* __restrict__ info, int halo) {
    using Tb = Tables<L>;
    Coord c;
    c.x[0] = blockIdx.x * blockDim.x + threadIdx.x;
    c.x[1] = blockIdx.y * blockDim.y + threadIdx.y;
    c.x[2] = blockIdx.z;
    if (c.x[0] >= geo.n[0] || c.x[1] >= geo.n[1]) return;
    auto cell_of = [&](const int* x) -> long long {
        int b[3];
        for (int a = 0; a < 3; ++a) b[a] = wrap_or_ghost(x[a], geo.n[a], geo.g[a], geo.periodic[a]);
        if (L::kDims == 2) b[2] = 0;
        return (long long)b[0] + (long long)geo.a[0] * (b[1] + (long long)geo.a[1] * b[2]);
    };
    const long long self = cell_of(c.x);
    uint32_t v = info[self];
    if (!(v & kInfoPresent)) return;
#pragma unroll
    for (int q = 1; q < L::kQ; ++q) {
        const int s[3] = {c.x[0] - Tb::cx(q), c.x[1] - Tb::cy(q), c.x[2] - Tb::cz(q)};
        bool missing = false;
        for (int a = 0; a < L::kDims; ++a) {
            if (geo.periodic[a]) continue;
            if ((s[a] < 0 && !((halo >> (2 * a)) & 1)) || (s[a] >= geo.n[a] && !((halo >> (2 * a + 1)) & 1)))
                missing = true;
        }
        if (!missing) missing = !(info[cell_of(s)] & kInfoPresent);
        if (missing) v |= 1u << q;
    }
    v |= (uint32_t)on_faces(geo, c, L::kDims) << kInfoFaceShift;
    info[self] = v;
}

void launch_node_info(int dims, const LevelGeom& geo, uint32_t* info, cudaStream_t s, int halo_faces) {
    dim3 g, b;
    step_shape(geo, dims, g, b);
    if (dims == 2)
        node_info_kernel<D2Q9><<<g, b, 0, s>>>(geo, info, halo_faces);
    else
        node_info_kernel<D3Q19><<<g, b, 0, s>>>(geo, info, halo_faces);
}

template <class S>
__global__ void fill_kernel(S* __restrict__ f, long long stride, int q, StepParams p, const double* __restrict__ value) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= stride) return;
    for (int k = 0; k < q; ++k) Storage<S>::store(f + k * stride + i, (typename Storage<S>::T)value[k], p);
}

cudaError_t launch_fill(int storage, void* f, long long stride, int q, const StepParams& p, const double* value,
                        cudaStream_t s) {
    const unsigned blocks = (unsigned)((stride + 255) / 256);
    switch (storage) {
        case 0: fill_kernel<double><<<blocks, 256, 0, s>>>((double*)f, stride, q, p, value); break;
        case 1: fill_kernel<float><<<blocks, 256, 0, s>>>((float*)f, stride, q, p, value); break;
        case 2: fill_kernel<__half><<<blocks, 256, 0, s>>>((__half*)f, stride, q, p, value); break;
        default: fill_kernel<__nv_bfloat16><<<blocks, 256, 0, s>>>((__nv_bfloat16*)f, stride, q, p, value); break;
    }
    return cudaGetLastError();
}

__global__ void conservation_final_kernel(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
    if (threadIdx.x < 4) {
        double v = 0.;
        for (int b = 0; b < nblocks; ++b) v += partial[b * 4 + threadIdx.x];
        out[threadIdx.x] = v;
    }
}

// ---------------------------------------------------------------- Morton neighbours
ZL_HD uint64_t axis_mask(int dims, int axis) {
    return dims == 2 ? (0x5555555555555555ull << axis) : (0x1249249249249249ull << axis);
}

ZL_HD uint64_t others_mask(int dims, int axis) {
    uint64_t m = 0;
    for (int a = 0; a < dims; ++a)
        if (a != axis) m |= axis_mask(dims, a);
    return m;
}

// FindXNeg etc. (morton_aux.hpp:65-79, :184-201)
ZL_HD uint64_t morton_neg(uint64_t code, int dims, int axis) {
    const uint64_t mk = axis_mask(dims, axis);
    const uint64_t v = code & mk;
    if (v == 0) return code;
    return ((v - 1) & mk) | (code & others_mask(dims, axis));
}

// FindXPos etc. (morton_aux.hpp:86-95, :208-219)
ZL_HD uint64_t morton_pos(uint64_t code, int dims, int axis) {
    const uint64_t mk = axis_mask(dims, axis);
    const uint64_t t = (code | ~mk) + 1;
    return (t & mk) | (code & others_mask(dims, axis));
}

__global__ void morton_neighbors_kernel(const uint64_t* __restrict__ codes, long long n, int dims,
                                        uint64_t* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t c = codes[i];
    for (int a = 0; a < dims; ++a) {
        out[i * 2 * dims + 2 * a] = morton_neg(c, dims, a);
        out[i * 2 * dims + 2 * a + 1] = morton_pos(c, dims, a);
    }
}

template <class L>
__global__ void upstream_index_kernel(const uint64_t* __restrict__ sorted, const long long* __restrict__ order,
                                      long long n, long long* __restrict__ out) {
    using Tb = Tables<L>;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t code = sorted[i];
    const long long node = order[i];
    for (int q = 0; q < L::kQ; ++q) {
        // upstream x - c_q: a Pos step where c < 0, a Neg step where c > 0, x then y then z
        uint64_t u = code;
        const int c[3] = {Tb::cx(q), Tb::cy(q), Tb::cz(q)};
        for (int a = 0; a < L::kDims; ++a) {
            if (c[a] > 0) u = morton_neg(u, L::kDims, a);
            if (c[a] < 0) u = morton_pos(u, L::kDims, a);
        }
        long long lo = 0, hi = n - 1, hit = -1;
        while (lo <= hi) {
            const long long mid = (lo + hi) >> 1;
            const uint64_t v = sorted[mid];
            if (v == u) {
                hit = order[mid];
                break;
            }
            if (v < u) lo = mid + 1;
            else hi = mid - 1;
        }
        out[node * L::kQ + q] = hit;
    }
}

cudaError_t launch_morton_neighbors(const uint64_t* codes, long long n, int dims, uint64_t* out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    morton_neighbors_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(codes, n, dims, out);
    return cudaGetLastError();
}

cudaError_t launch_upstream_index(int dims, const uint64_t* sorted, const long long* order, long long n,
                                  long long* out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (dims == 2)
        upstream_index_kernel<D2Q9><<<blocks, 256, 0, s>>>(sorted, order, n, out);
    else
        upstream_index_kernel<D3Q19><<<blocks, 256, 0, s>>>(sorted, order, n, out);
    return cudaGetLastError();
}

cudaError_t launch_decode_minmax(const uint64_t* codes, long long n, int dims, int* minmax, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    decode_minmax_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(codes, n, dims, minmax);
    return cudaGetLastError();
}

cudaError_t launch_mark_present(const uint64_t* codes, long long n, const LevelMap& m, const LevelGeom& geo,
                                uint32_t* info, int* bad, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    mark_present_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(codes, n, m, geo, info, bad);
    return cudaGetLastError();
}

// every node of the box is present (ghost frame cells stay absent)
__global__ void mark_box_kernel(LevelGeom geo, uint32_t* __restrict__ info) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nn = (long long)geo.n[0] * geo.n[1] * geo.n[2];
    if (i >= nn) return;
    const long long x = i % geo.n[0], r = i / geo.n[0], y = r % geo.n[1], z = r / geo.n[1];
    const long long cell = (x + geo.g[0]) + (long long)geo.a[0] * ((y + geo.g[1]) + (long long)geo.a[1] * (z + geo.g[2]));
    info[cell] = kInfoPresent;
}

cudaError_t launch_mark_box(const LevelGeom& geo, uint32_t* info, cudaStream_t s) {
    const long long nn = (long long)geo.n[0] * geo.n[1] * geo.n[2];
    mark_box_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(geo, info);
    return cudaGetLastError();
}

cudaError_t launch_count_present(const uint32_t* info, long long cells, unsigned long long* count, cudaStream_t s) {
    const long long blocks = std::min<long long>((cells + 255) / 256, 148 * 8);
    count_present_kernel<<<(unsigned)std::max<long long>(blocks, 1), 256, 0, s>>>(info, cells, count);
    return cudaGetLastError();
}


// Indices i < n with mark[i] != 0, ascending, into out; *count (device) gets their number.
// With tmp == nullptr only *tmp_bytes is set.
cudaError_t select_marked(const uint32_t* mark, int n, int* out, int* count, void* tmp, size_t* tmp_bytes,
                          cudaStream_t s) {
    return cub::DeviceSelect::Flagged(tmp, *tmp_bytes, thrust::counting_iterator<int>(0), mark, out, count, n, s);
}

cudaError_t sort_pairs_by_key(const int* keys_in, int* keys_out, const int* vals_in, int* vals_out, int n, int key_bits,
                              void* tmp, size_t* tmp_bytes, cudaStream_t s) {
    return cub::DeviceRadixSort::SortPairs(tmp, *tmp_bytes, keys_in, keys_out, vals_in, vals_out, n, 0, key_bits, s);
}

}  // namespace zl
