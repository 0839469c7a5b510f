// Device side of the VTK XML field output (vtu.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace zl {

// One level's points in output order and the bounding box of their level indices.
struct VtuLevel {
    const uint64_t* codes;  // reference Morton codes at this level
    const int32_t* flags;   // flag_status per point
    long long n;
    int dims, level;
    double space[3];        // background grid spacing
    double origin[3];       // coordinate of level index 0
    uint32_t ghost_mask;    // flag bits written as vtkGhostType 1
    long long lo[3], ext[3];  // index box of the point table
};

cudaError_t vtu_points(const VtuLevel& a, const double* rho, const double* u, uint16_t* flag_out, uint8_t* ghost_out,
                       float* rho_out, float* u_out, float* xyz, int32_t* table, cudaStream_t s);
size_t vtu_scan_bytes(long long n);
cudaError_t vtu_cells(const VtuLevel& a, const int32_t* table, uint32_t* is_cell, uint32_t* first, void* scan_tmp,
                      size_t scan_bytes, cudaStream_t s);
cudaError_t vtu_connect(const VtuLevel& a, const int32_t* table, const uint32_t* is_cell, const uint32_t* first,
                        uint64_t* conn, cudaStream_t s);
cudaError_t vtu_offsets(long long cells, int dims, uint64_t* offsets, uint8_t* types, cudaStream_t s);
unsigned long long base64_chars(unsigned long long nbytes);
cudaError_t base64_encode(const void* payload, unsigned long long nbytes, char* out, cudaStream_t s);

}  // namespace zl
