// FP64 population storage, reference arithmetic order.  Built with -fmad=false.
#include "launch.cuh"
namespace zl {
ZL_DEFINE_LAUNCH_SET(launch_set_f64, double)
}  // namespace zl
