// stage3d_zm_euler_fp64.cu -- the z-marching 3D stage kernel (stage3d_zm.cuh) for
// Euler stages in the FP64 form; one unit per (integrator, form) so the
// instantiations compile in parallel.
#include "kernels.cuh"

namespace smaug {

#include "stage3d_zm.cuh"

SMAUG_ZM_UNIT(SMAUG_INT_EULER, false, euler_fp64)

}  // namespace smaug
