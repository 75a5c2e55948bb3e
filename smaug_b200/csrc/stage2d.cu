// stage2d.cu -- translation unit of the 2D stage kernel (stage2d.cuh)
// and its launch dispatcher.
#include "kernels.cuh"

namespace smaug {

#include "stage2d.cuh"

cudaError_t launch_stage2d_any(int mode, bool mix, const KParams& K, const KBufs& B, cudaStream_t st) {
  if (mode == SMAUG_INT_EULER)
    return mix ? launch_stage2d<SMAUG_INT_EULER, true>(K, B, st) : launch_stage2d<SMAUG_INT_EULER, false>(K, B, st);
  return mix ? launch_stage2d<SMAUG_INT_RK4, true>(K, B, st) : launch_stage2d<SMAUG_INT_RK4, false>(K, B, st);
}

cudaError_t stage2d_set_attributes() {
  cudaError_t e;
  if ((e = stage2d_attr<SMAUG_INT_EULER, true, false>())) return e;
  if ((e = stage2d_attr<SMAUG_INT_EULER, false, false>())) return e;
  if ((e = stage2d_attr<SMAUG_INT_RK4, true, false>())) return e;
  if ((e = stage2d_attr<SMAUG_INT_RK4, false, false>())) return e;
  if ((e = stage2d_attr<SMAUG_INT_EULER, true, true>())) return e;
  if ((e = stage2d_attr<SMAUG_INT_EULER, false, true>())) return e;
  if ((e = stage2d_attr<SMAUG_INT_RK4, true, true>())) return e;
  return stage2d_attr<SMAUG_INT_RK4, false, true>();
}

}  // namespace smaug
