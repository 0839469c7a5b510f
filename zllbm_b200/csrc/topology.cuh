// Declarations of the topology and set-up launchers (topology.cu).
#pragma once
#include <algorithm>
#include "launch.cuh"

namespace zl {

ZL_HD uint64_t morton_neg(uint64_t code, int dims, int axis);
ZL_HD uint64_t morton_pos(uint64_t code, int dims, int axis);

cudaError_t launch_decode_minmax(const uint64_t* codes, long long n, int dims, int* minmax, cudaStream_t s);
cudaError_t launch_mark_present(const uint64_t* codes, long long n, const LevelMap& m, const LevelGeom& geo,
                                uint32_t* info, int* bad, cudaStream_t s);
cudaError_t launch_count_present(const uint32_t* info, long long cells, unsigned long long* count, cudaStream_t s);
cudaError_t launch_mark_box(const LevelGeom& geo, uint32_t* info, cudaStream_t s);
void launch_node_info(int dims, const LevelGeom& geo, uint32_t* info, cudaStream_t s, int halo_faces = 0);
cudaError_t launch_fill(int storage, void* f, long long stride, int q, const StepParams& p, const double* value,
                        cudaStream_t s);
cudaError_t launch_morton_neighbors(const uint64_t* codes, long long n, int dims, uint64_t* out, cudaStream_t s);
cudaError_t launch_upstream_index(int dims, const uint64_t* sorted, const long long* order, long long n,
                                  long long* out, cudaStream_t s);
// Stable radix sort of (key, value) pairs on the low key_bits bits of the keys (null tmp: size query).
cudaError_t sort_pairs_by_key(const int* keys_in, int* keys_out, const int* vals_in, int* vals_out, int n, int key_bits,
                              void* tmp, size_t* tmp_bytes, cudaStream_t s);
cudaError_t select_marked(const uint32_t* mark, int n, int* out, int* count, void* tmp, size_t* tmp_bytes,
                          cudaStream_t s);

}  // namespace zl
