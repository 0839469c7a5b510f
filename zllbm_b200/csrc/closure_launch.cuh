// Host-side entry points of the closure and full-box kernels (closure.cu) used by the API.
#pragma once
#include <cuda_runtime.h>

#include "aa_kernel.cuh"

namespace zl {

enum ClosureBoxOp { kBoxSetEq = 0, kBoxGetMacros = 1, kBoxFeatures = 2, kBoxFilter = 3 };

// Full-box level kernels over the populations f (storage F32 / F16 / BF16):
//   kBoxSetEq      a = rho, b = u                 -> f = feq(rho, u)
//   kBoxGetMacros  b = rho, c = u
//   kBoxFeatures   b = closure features (n x 24)
//   kBoxFilter     b = factor^3 block means (nc[0] nc[1] nc[2] x 29)
cudaError_t closure_box_op(int op, int storage, void* f, const LevelGeom& geo, const StepParams& p, int even,
                           const float* a, float* b, float* c, int factor, const int* nc, cudaStream_t s);

// One AA step of a full periodic D3Q19 box with the learned closure in the collision
// (net: device zl_mlp; fallback_c: Smagorinsky c used where the network output is not finite;
// c_node: per-cell c written for the steps that reuse it, or nullptr).
cudaError_t closure_learned_step(int storage, int coll, bool odd, void* f, const LevelGeom& geo, const StepParams& p,
                                 const float* net, float fallback_c, float* c_node, int* err, cudaStream_t s);

}  // namespace zl
