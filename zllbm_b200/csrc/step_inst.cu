// One part of the fused step launchers of a (storage, lattice, collision): ZL_STEP_PART 0 / 1 is
// the even / odd step of the AA pattern, 2 .. 5 the batched multi-level step with extensions
// 0, force, LES, force + LES.  The build compiles this file once per combination with ZL_STEP_S
// (storage type), ZL_STEP_L (lattice), ZL_STEP_C (collision) and ZL_STEP_PART defined; the FP64
// storage with -fmad=false, like every FP64 kernel, so its arithmetic follows the reference's
// rounding step for step.
#include "step_launch.cuh"

#if !defined(ZL_STEP_S) || !defined(ZL_STEP_L) || !defined(ZL_STEP_C) || !defined(ZL_STEP_PART)
#error "step_inst.cu needs ZL_STEP_S, ZL_STEP_L, ZL_STEP_C and ZL_STEP_PART"
#endif

namespace zl {
#if ZL_STEP_PART < 2
template cudaError_t step_lco<ZL_STEP_S, ZL_STEP_L, ZL_STEP_C, ZL_STEP_PART == 1>(bool, bool, ZL_STEP_S*,
                                                                                  const LevelGeom&, const StepParams&,
                                                                                  cudaStream_t);
#else
template cudaError_t batch_lcx<ZL_STEP_S, ZL_STEP_L, ZL_STEP_C, ZL_STEP_PART - 2>(const LevelBatch&, cudaStream_t);
#endif
}  // namespace zl
