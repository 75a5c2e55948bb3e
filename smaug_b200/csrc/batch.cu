// batch.cu -- the batched 2D stage kernel (batch_kernel.cuh) at the 32x8
// tile of the single-run kernel.
#include "kernels.cuh"

namespace smaug {
namespace t32x8 {

#include "stage2d.cuh"
#include "batch_kernel.cuh"

}  // namespace t32x8
}  // namespace smaug
