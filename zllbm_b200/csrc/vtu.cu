// Field output in the reference's VTK XML layout, built on the device: per level the point
// arrays (flag_status, vtkGhostType, rho, velocity, coordinates), the cell connectivity and the
// base64 text of each binary array (amr_project/io/vtk_writer_manager.cpp:29-77, :374-1235).
#include <cub/cub.cuh>
#include "vtu.cuh"
#include "level_ops.cuh"

namespace zl {

namespace {

__device__ __forceinline__ long long table_index(const VtuLevel& a, const long long* idx) {
    long long t = 0;
    for (int d = a.dims - 1; d >= 0; --d) {
        const long long v = idx[d] - a.lo[d];
        if (v < 0 || v >= a.ext[d]) return -1;
        t = t * a.ext[d] + v;
    }
    return t;
}

// one thread per point: output arrays and the point's index in the table of its level cell
__global__ void vtu_points_kernel(VtuLevel a, const double* __restrict__ rho, const double* __restrict__ u,
                                  uint16_t* __restrict__ flag_out, uint8_t* __restrict__ ghost_out,
                                  float* __restrict__ rho_out, float* __restrict__ u_out, float* __restrict__ xyz,
                                  int32_t* __restrict__ table) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const uint64_t code = a.codes[i];
    const int32_t flag = a.flags[i];
    flag_out[i] = (uint16_t)flag;
    ghost_out[i] = (flag & (int32_t)a.ghost_mask) != 0 ? 1 : 0;
    rho_out[i] = (float)rho[i];
    for (int d = 0; d < a.dims; ++d) u_out[i * a.dims + d] = (float)u[i * a.dims + d];
    // SFBitsetComputeCoordinate (morton_aux.cpp:86-101, :310-333): origin, then the level spacing
    // times 2^bit for every set bit of the axis, bits in ascending order
    for (int d = 0; d < 3; ++d) {
        double c = 0.;
        if (d < a.dims) {
            const double gs = a.space[d] / (double)(1ull << a.level);
            c = a.origin[d];
            for (int b = 0; b < 64 / a.dims; ++b)
                if ((code >> (a.dims * b + d)) & 1ull) c += gs * (double)(1ull << b);
        }
        xyz[i * 3 + d] = (float)c;
    }
    uint32_t idx[3];
    morton_decode(code, a.dims, idx);
    const long long li[3] = {idx[0], idx[1], idx[2]};
    const long long t = table_index(a, li);
    if (t >= 0) table[t] = (int32_t)i;
}

__device__ __forceinline__ bool cell_corners(const VtuLevel& a, const int32_t* table, long long i, int32_t* pts) {
    uint32_t idx[3];
    morton_decode(a.codes[i], a.dims, idx);
    // corner k sits at (+x, +y, +z) = bits 0, 1, 2 of k: (0,0,0), (+x), (+y), (+x,+y), (+z), ...
    const int corners = a.dims == 2 ? 4 : 8;
    for (int k = 0; k < corners; ++k) {
        const long long li[3] = {(long long)idx[0] + (k & 1), (long long)idx[1] + ((k >> 1) & 1),
                                 (long long)idx[2] + ((k >> 2) & 1)};
        const long long t = table_index(a, li);
        if (t < 0) return false;
        pts[k] = table[t];
        if (pts[k] < 0) return false;
    }
    return true;
}

// SFBitsetBelongToOneCell (sfbitset_aux.h:738-830): a point starts a cell when all corners exist
__global__ void vtu_cell_flag_kernel(VtuLevel a, const int32_t* __restrict__ table, uint32_t* __restrict__ is_cell) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    int32_t pts[8];
    is_cell[i] = cell_corners(a, table, i, pts) ? 1u : 0u;
}

__global__ void vtu_connect_kernel(VtuLevel a, const int32_t* __restrict__ table, const uint32_t* __restrict__ is_cell,
                                   const uint32_t* __restrict__ first, uint64_t* __restrict__ conn) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= a.n || !is_cell[i]) return;
    int32_t pts[8];
    cell_corners(a, table, i, pts);
    const int corners = a.dims == 2 ? 4 : 8;
    for (int k = 0; k < corners; ++k) conn[(long long)first[i] * corners + k] = (uint64_t)pts[k];
}

__global__ void vtu_offsets_kernel(long long cells, int corners, uint8_t type, uint64_t* __restrict__ offsets,
                                   uint8_t* __restrict__ types) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= cells) return;
    offsets[i] = (uint64_t)(i + 1) * (uint64_t)corners;
    types[i] = type;
}

// Base64 of [UInt32 byte count][payload] (Base64Utility::Encode): thread g encodes input bytes
// 3g .. 3g + 2 of that stream into four characters, '=' padding the last group.
__constant__ char kB64[65] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";

__global__ void base64_kernel(const uint8_t* __restrict__ payload, unsigned long long nbytes, uint32_t header,
                              char* __restrict__ out) {
    const unsigned long long total = nbytes + 4;
    const unsigned long long g = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    const unsigned long long groups = (total + 2) / 3;
    if (g >= groups) return;
    uint32_t b[3];
    const unsigned long long s = 3 * g;
    int have = 0;
    for (int k = 0; k < 3; ++k) {
        const unsigned long long j = s + k;
        if (j < total) {
            b[k] = j < 4 ? (header >> (8 * j)) & 0xffu : payload[j - 4];
            ++have;
        } else {
            b[k] = 0;
        }
    }
    char4 o;
    o.x = kB64[(b[0] >> 2) & 0x3f];
    o.y = kB64[((b[0] << 4) & 0x30) | ((b[1] >> 4) & 0x0f)];
    o.z = have > 1 ? kB64[((b[1] << 2) & 0x3c) | ((b[2] >> 6) & 0x03)] : '=';
    o.w = have > 2 ? kB64[b[2] & 0x3f] : '=';
    reinterpret_cast<char4*>(out)[g] = o;
}

unsigned grid_of(long long n, int block) { return (unsigned)((n + block - 1) / block); }

}  // namespace

cudaError_t vtu_points(const VtuLevel& a, const double* rho, const double* u, uint16_t* flag_out, uint8_t* ghost_out,
                       float* rho_out, float* u_out, float* xyz, int32_t* table, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    vtu_points_kernel<<<grid_of(a.n, 256), 256, 0, s>>>(a, rho, u, flag_out, ghost_out, rho_out, u_out, xyz, table);
    return cudaGetLastError();
}

size_t vtu_scan_bytes(long long n) {
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)n);
    return bytes;
}

cudaError_t vtu_cells(const VtuLevel& a, const int32_t* table, uint32_t* is_cell, uint32_t* first, void* scan_tmp,
                      size_t scan_bytes, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    vtu_cell_flag_kernel<<<grid_of(a.n, 256), 256, 0, s>>>(a, table, is_cell);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, is_cell, first, (int)a.n, s);
}

cudaError_t vtu_connect(const VtuLevel& a, const int32_t* table, const uint32_t* is_cell, const uint32_t* first,
                        uint64_t* conn, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    vtu_connect_kernel<<<grid_of(a.n, 256), 256, 0, s>>>(a, table, is_cell, first, conn);
    return cudaGetLastError();
}

cudaError_t vtu_offsets(long long cells, int dims, uint64_t* offsets, uint8_t* types, cudaStream_t s) {
    if (cells <= 0) return cudaSuccess;
    // VTK_PIXEL (8) with 4 corners in 2D, VTK_VOXEL (11) with 8 in 3D (WriteGridCellTypes / Offsets)
    vtu_offsets_kernel<<<grid_of(cells, 256), 256, 0, s>>>(cells, dims == 2 ? 4 : 8, dims == 2 ? 8 : 11, offsets,
                                                          types);
    return cudaGetLastError();
}

unsigned long long base64_chars(unsigned long long nbytes) { return (nbytes + 4 + 2) / 3 * 4; }

cudaError_t base64_encode(const void* payload, unsigned long long nbytes, char* out, cudaStream_t s) {
    const unsigned long long groups = (nbytes + 4 + 2) / 3;
    if (nbytes > 0xffffffffull) return cudaErrorInvalidValue;
    base64_kernel<<<grid_of((long long)groups, 256), 256, 0, s>>>(static_cast<const uint8_t*>(payload), nbytes,
                                                                 (uint32_t)nbytes, out);
    return cudaGetLastError();
}

}  // namespace zl
