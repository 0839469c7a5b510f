// FP32 deviation storage (f - w), FP32 collision.
#include "launch.cuh"
namespace zl {
ZL_DEFINE_LAUNCH_SET(launch_set_f32, float)
}  // namespace zl
