// stage2d_tma.cu -- the 2D stage kernel with its tiles staged by bulk tensor
// copies (TMA).
//
// The stage body is stage2d.cuh's, compiled here with its own region
// constants: the staged region of a 32x8 tile is 40 cells wide (3 halo
// columns on the left, 5 on the right) so that a row is 320 bytes (FP64) or
// 160 bytes (float), a multiple of the copy's 16-byte granule, and tile
// column bx starts at x = 3 + 32 (bx - 1), so that the region's first
// column 32 (bx - 1) is a multiple of 32 cells (the copy's x offset must be
// 16-byte aligned).  Tile column 0 holds only the interior column x = 2.
//
// One thread issues the copies of a tile -- the 6 fields of the stage input
// as one box [6][14][40], and the 4 background fields (or rho_b alone) as a
// second box -- completing on the block's mbarrier.  Two launch forms: one
// block per tile, or a persistent grid (resident blocks per SM x SMs; block
// b owns the tiles b, b + grid, ...).  In the persistent form a block copies
// its next tile as soon as the current tile's staged arrays are dead (after
// the last hyperdiffusion pass and the reads of its combine), overlapping
// the copy with the tile's stores, ghost images and CFL epilogue; the mixed
// form without background fields, where a second state buffer still fits 4
// blocks per SM, copies the next tile's state into the other buffer a whole
// tile ahead and its rho_b during the stores (two arrivals per phase).
// Cells outside the grid read 0 (the copy's fill value), as the per-thread
// staging stores them.  Every wait on the mbarrier is bounded (TMA_WAIT_NS);
// a block whose copy does not arrive sets FLAG_TMA_TIMEOUT, waits (bounded)
// for its copies in flight and exits.
//
// The arithmetic is the per-thread-staged kernel's, cell for cell, so the
// kernels' results are bitwise identical.  On B200 at 4096^2 these kernels
// run about 10 % slower than the per-thread staging (RK4 FP64 11.4 vs 10.5 ms
// per step, mixed 10.5 vs 9.5), which therefore stays the engine's default.
#include <cuda.h>

#include "kernels.cuh"

namespace smaug {
namespace tma {

constexpr int TX = 32, TY = 8;
constexpr int RX = TX + 8;  // 3 + 32 + 5 columns: 16-byte-multiple rows in float and double
constexpr int RY = TY + 2 * HALO;
constexpr int RC = RX * RY;
constexpr int RXU = RX;  // all 40 columns (the last two are never read; skipping them in the
                        // region loops measured more shared-memory bank conflicts)
constexpr int NTHREADS = TX * TY;
constexpr int XORG = 3 - TX;  // tile column bx starts at 3 + TX (bx - 1)
static_assert((XORG - HALO) % 32 == 0, "region start must be a multiple of 32 cells");
static_assert(RX * sizeof(float) % 16 == 0 && RX * sizeof(double) % 16 == 0, "row of a copy box");

#include "stage2d.cuh"

// the staging of a specialisation: two state buffers where they keep 4
// blocks per SM (the mixed form without background fields), else one
template <bool BG, bool MIX>
__host__ __device__ constexpr int tma_form() {
  return (!BG && MIX) ? 2 : 1;
}

template <int MODE, bool BG, bool MIX>
__global__ void __launch_bounds__(NTHREADS, SMAUG_MINB2D)
    stage2d_tma_kernel(const KParams P, const KBufs B, const __grid_constant__ CUtensorMap ms,
                       const __grid_constant__ CUtensorMap mg, int nbx, int ntiles) {
  __shared__ unsigned long long bar;
  // arrivals per phase: the copy of the state and, with two state buffers,
  // the separate copy of rho_b
  if (threadIdx.x == 0 && threadIdx.y == 0) mbar_init(&bar, tma_form<BG, MIX>());
  __syncthreads();
  TmaTile tt{&ms, &mg, &bar, 0u, true, -1, 0};
  unsigned k = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, k++) {
    const int next = tile + (int)gridDim.x;
    tt.parity = k & 1u;
    tt.issue_self = k == 0;
    tt.nbx = next < ntiles ? next % nbx : -1;
    tt.nby = next / nbx;
    if (!stage2d_body<MODE, BG, MIX, false, false, tma_form<BG, MIX>()>(P, B, tile % nbx, tile / nbx, &tt))
      return;
  }
}

// dynamic shared memory: the stage body's layout plus alignment slack (the
// body rounds its base up to 128 bytes for the copies)
template <bool BG, bool MIX>
constexpr size_t tma_smem() {
  return s2::smem_bytes<BG, MIX, false>() + 128 +
         (tma_form<BG, MIX>() == 2 ? 6 * RC * sizeof(typename Form<MIX>::S) : 0);
}

template <int MODE, bool BG, bool MIX>
static cudaError_t tma_attr(int* bps) {
  auto k = stage2d_tma_kernel<MODE, BG, MIX>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tma_smem<BG, MIX>());
  if (e) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k, NTHREADS, tma_smem<BG, MIX>());
}

// resident blocks per SM, [bg][mix] (the smaller of the two modes)
static int g_bps[2][2] = {{0, 0}, {0, 0}};

}  // namespace tma

bool stage2d_tma_supported(const KParams& K, bool mix) {
  if (K.order6 || K.n2 != 1) return false;
  const long es = mix ? 4 : 8;
  // row pitch of the stage input and of the background fields (double)
  return ((long)K.n0 * es) % 16 == 0 && ((long)K.n0 * 8) % 16 == 0 && K.n0 >= 5 && K.n1 >= 5;
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// the driver's tensor-map encoder, looked up once (a function-local static
// is initialised once even when engines are created from several threads)
static EncodeTiled encode_tiled() {
  static const EncodeTiled fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<EncodeTiled>(p);
    cudaGetLastError();
    return static_cast<EncodeTiled>(nullptr);
  }();
  return fn;
}

int stage2d_tma_encode(TmaMap* m, const void* base, bool f32, const KParams& K, int nfield, int box_fields) {
  static_assert(sizeof(TmaMap) == sizeof(CUtensorMap) && alignof(TmaMap) >= alignof(CUtensorMap),
                "TmaMap holds a CUtensorMap");
  EncodeTiled fn = encode_tiled();
  if (!fn || !base || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return 1;
  const cuuint64_t es = f32 ? 4 : 8;
  const cuuint64_t dim[3] = {(cuuint64_t)K.n0, (cuuint64_t)K.n1, (cuuint64_t)nfield};
  const cuuint64_t stride[2] = {(cuuint64_t)K.n0 * es, (cuuint64_t)K.n0 * (cuuint64_t)K.n1 * es};
  const cuuint32_t box[3] = {(cuuint32_t)tma::RX, (cuuint32_t)tma::RY, (cuuint32_t)box_fields};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = fn(reinterpret_cast<CUtensorMap*>(m),
                        f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                        const_cast<void*>(base), dim, stride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : 1;
}

cudaError_t stage2d_tma_set_attributes() {
  cudaError_t e;
#define SMAUG_TMA_ATTR(BG, MIX)                                              \
  {                                                                          \
    int b0 = 0, b1 = 0;                                                      \
    if ((e = tma::tma_attr<SMAUG_INT_EULER, BG, MIX>(&b0))) return e;        \
    if ((e = tma::tma_attr<SMAUG_INT_RK4, BG, MIX>(&b1))) return e;          \
    tma::g_bps[BG][MIX] = b0 < b1 ? b0 : b1;                                 \
  }
  SMAUG_TMA_ATTR(false, false)
  SMAUG_TMA_ATTR(false, true)
  SMAUG_TMA_ATTR(true, false)
  SMAUG_TMA_ATTR(true, true)
#undef SMAUG_TMA_ATTR
  return cudaSuccess;
}

cudaError_t launch_stage2d_tma(int mode, bool mix, const KParams& K, const KBufs& B, const TmaMap& ms,
                               const TmaMap& mg, bool persistent, cudaStream_t st) {
  using tma::stage2d_tma_kernel;
  using tma::tma_smem;
  const int nbx = (K.n0 - 3 - tma::XORG) / tma::TX + 1, nby = (K.n1 - 4 + tma::TY - 1) / tma::TY;
  const int ntiles = nbx * nby;
  int dev = 0, nsm = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev)) || (e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)))
    return e;
  const bool bg = K.has_bg != 0;
  int bps = tma::g_bps[bg][mix];
  if (bps < 1) bps = 1;
  const int grid = (persistent && bps * nsm < ntiles) ? bps * nsm : ntiles;
  const CUtensorMap& m0 = *reinterpret_cast<const CUtensorMap*>(&ms);
  const CUtensorMap& m1 = *reinterpret_cast<const CUtensorMap*>(&mg);
  const dim3 block(tma::TX, tma::TY);
#define SMAUG_TMA_LAUNCH(M, BG, MIX) \
  stage2d_tma_kernel<M, BG, MIX><<<grid, block, tma_smem<BG, MIX>(), st>>>(K, B, m0, m1, nbx, ntiles)
  if (mode == SMAUG_INT_EULER) {
    if (bg) {
      if (mix) SMAUG_TMA_LAUNCH(SMAUG_INT_EULER, true, true); else SMAUG_TMA_LAUNCH(SMAUG_INT_EULER, true, false);
    } else {
      if (mix) SMAUG_TMA_LAUNCH(SMAUG_INT_EULER, false, true); else SMAUG_TMA_LAUNCH(SMAUG_INT_EULER, false, false);
    }
  } else {
    if (bg) {
      if (mix) SMAUG_TMA_LAUNCH(SMAUG_INT_RK4, true, true); else SMAUG_TMA_LAUNCH(SMAUG_INT_RK4, true, false);
    } else {
      if (mix) SMAUG_TMA_LAUNCH(SMAUG_INT_RK4, false, true); else SMAUG_TMA_LAUNCH(SMAUG_INT_RK4, false, false);
    }
  }
#undef SMAUG_TMA_LAUNCH
  return cudaGetLastError();
}

}  // namespace smaug
