// FP16 / BF16 scaled deviation storage, FP32 collision.
#include "launch.cuh"
namespace zl {
ZL_DEFINE_LAUNCH_SET(launch_set_f16, __half)
ZL_DEFINE_LAUNCH_SET(launch_set_bf16, __nv_bfloat16)
}  // namespace zl
