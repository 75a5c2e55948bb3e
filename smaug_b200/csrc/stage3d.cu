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

cudaError_t stage3d_set_attributes() {
  cudaError_t e;
#define SMAUG_ATTR3(M, BG, MIX)                                              \
  if ((e = stage3d_attr<M, BG, MIX, false>())) return e;                   \
  if ((e = stage3d_attr<M, BG, MIX, true>())) return e;
  SMAUG_ATTR3(SMAUG_INT_EULER, true, false)
  SMAUG_ATTR3(SMAUG_INT_EULER, false, false)
  SMAUG_ATTR3(SMAUG_INT_RK4, true, false)
  SMAUG_ATTR3(SMAUG_INT_RK4, false, false)
  SMAUG_ATTR3(SMAUG_INT_EULER, true, true)
  SMAUG_ATTR3(SMAUG_INT_EULER, false, true)
  SMAUG_ATTR3(SMAUG_INT_RK4, true, true)
  SMAUG_ATTR3(SMAUG_INT_RK4, false, true)
#undef SMAUG_ATTR3
  return cudaSuccess;
}

}  // namespace smaug
