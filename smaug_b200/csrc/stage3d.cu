// stage3d.cu -- launch dispatcher of the 3D stage kernel: the z-marching
// kernel of stage3d_zm.cuh, instantiated per integrator and precision form
// by stage3d_zm_{euler,rk4}_{fp64,mixed}.cu.
#include <atomic>

#include "kernels.cuh"

namespace smaug {

// SM count of the current device (the z-chunk length depends on it), looked
// up once per device
static int sm_count() {
  static std::atomic<int> cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  int v = cache[dev].load(std::memory_order_relaxed);
  if (v <= 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    cache[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}

cudaError_t launch_stage3d_any(int mode, bool mix, const KParams& K, const KBufs& B, cudaStream_t st) {
  const int nsm = sm_count();
  if (mode == SMAUG_INT_EULER)
    return mix ? zm_launch_euler_mixed(K, B, st, nsm) : zm_launch_euler_fp64(K, B, st, nsm);
  return mix ? zm_launch_rk4_mixed(K, B, st, nsm) : zm_launch_rk4_fp64(K, B, st, nsm);
}

cudaError_t stage3d_set_attributes() {
  cudaError_t e;
  if ((e = zm_attr_euler_fp64())) return e;
  if ((e = zm_attr_euler_mixed())) return e;
  if ((e = zm_attr_rk4_fp64())) return e;
  return zm_attr_rk4_mixed();
}

}  // namespace smaug
