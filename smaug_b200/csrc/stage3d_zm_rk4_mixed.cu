// stage3d_zm_rk4_mixed.cu -- the z-marching 3D stage kernel (stage3d_zm.cuh) for
// RK4 stages in the mixed-precision form; one unit per (integrator, form) so the
// instantiations compile in parallel.
#include "kernels.cuh"

namespace smaug {

#include "stage3d_zm.cuh"

SMAUG_ZM_UNIT(SMAUG_INT_RK4, true, rk4_mixed)

}  // namespace smaug
