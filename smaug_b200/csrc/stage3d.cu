// stage3d.cu -- translation unit of the 3D stage kernel (stage3d.cuh)
// and its launch dispatcher.
#include "kernels.cuh"

namespace smaug {

#include "stage3d.cuh"

cudaError_t launch_stage3d_any(int mode, bool mix, const KParams& K, const KBufs& B, cudaStream_t st) {
  if (mode == SMAUG_INT_EULER)
    return mix ? launch_stage3d<SMAUG_INT_EULER, true>(K, B, st) : launch_stage3d<SMAUG_INT_EULER, false>(K, B, st);
  return mix ? launch_stage3d<SMAUG_INT_RK4, true>(K, B, st) : launch_stage3d<SMAUG_INT_RK4, false>(K, B, st);
}

}  // namespace smaug
