// stage3d_zm_euler_mixed.cu -- the z-marching 3D stage kernel (stage3d_zm.cuh) for
// Euler stages in the mixed-precision form; one unit per (integrator, form) so the
// instantiations compile in parallel.
#include "kernels.cuh"

namespace smaug {

#include "stage3d_zm.cuh"

SMAUG_ZM_UNIT(SMAUG_INT_EULER, true, euler_mixed)

}  // namespace smaug
