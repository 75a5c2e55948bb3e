// batch16.cu -- the batched 2D stage kernel (batch_kernel.cuh) at a 16x16
// tile: the same stage body with its own tile constants, one of the shapes
// the ensemble's autotuner times.
#include "kernels.cuh"

namespace smaug {
namespace t16x16 {

constexpr int TX = 16, TY = 16;
constexpr int RX = TX + 2 * HALO, RY = TY + 2 * HALO;
constexpr int RC = RX * RY;
constexpr int RXU = RX;
constexpr int NTHREADS = TX * TY;

#include "stage2d.cuh"
#include "batch_kernel.cuh"

}  // namespace t16x16
}  // namespace smaug
