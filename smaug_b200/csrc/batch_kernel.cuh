// batch_kernel.cuh -- the batched 2D stage kernel and its launch helpers,
// included after stage2d.cuh inside a namespace that fixes the tile shape
// (TX, TY and the derived region constants): batch.cu instantiates it for the
// 32x8 tile of the single-run kernel, batch16.cu for 16x16, and the
// ensemble's autotuner times both (engine.cu, batch_tune).
//
// Every run keeps its own parameter block, buffers, CFL maxima and dt; the
// tiles of all runs form one work list, and a persistent grid of blocks walks
// it (block i takes tiles i, i + grid, ...), calling the same stage body as
// the single-run kernel.  Runs of different sizes, boundary types, drivers and
// background fields share the launch; the background specialisation is
// always on (exact for runs without backgrounds too).
#pragma once

template <int MODE, bool MIX>
__global__ void __launch_bounds__(NTHREADS, SMAUG_MINB2D)
    stage2d_batch(const KParams* __restrict__ Ks, const KBufs* __restrict__ Bs,
                  const int4* __restrict__ tiles, int ntiles) {
  for (int it = blockIdx.x; it < ntiles; it += gridDim.x) {
    const int4 t = tiles[it];  // run, tile x, tile y
    stage2d_body<MODE, true, MIX>(Ks[t.x], Bs[t.x], t.y, t.z);
    __syncthreads();
  }
}

cudaError_t launch_batch2d(int mode, bool mix, const KParams* Ks, const KBufs* Bs, const int4* tiles,
                           int ntiles, int grid, cudaStream_t st) {
  const dim3 block(TX, TY);
  const size_t sm = mix ? s2::smem_bytes<true, true>() : s2::smem_bytes<true, false>();
  if (mode == SMAUG_INT_EULER) {
    if (mix)
      stage2d_batch<SMAUG_INT_EULER, true><<<grid, block, sm, st>>>(Ks, Bs, tiles, ntiles);
    else
      stage2d_batch<SMAUG_INT_EULER, false><<<grid, block, sm, st>>>(Ks, Bs, tiles, ntiles);
  } else {
    if (mix)
      stage2d_batch<SMAUG_INT_RK4, true><<<grid, block, sm, st>>>(Ks, Bs, tiles, ntiles);
    else
      stage2d_batch<SMAUG_INT_RK4, false><<<grid, block, sm, st>>>(Ks, Bs, tiles, ntiles);
  }
  return cudaGetLastError();
}

cudaError_t batch2d_set_attributes() {
  cudaError_t e;
  const int s64 = (int)s2::smem_bytes<true, false>(), s32 = (int)s2::smem_bytes<true, true>();
  if ((e = cudaFuncSetAttribute(stage2d_batch<SMAUG_INT_EULER, false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, s64)))
    return e;
  if ((e = cudaFuncSetAttribute(stage2d_batch<SMAUG_INT_RK4, false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, s64)))
    return e;
  if ((e = cudaFuncSetAttribute(stage2d_batch<SMAUG_INT_EULER, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, s32)))
    return e;
  return cudaFuncSetAttribute(stage2d_batch<SMAUG_INT_RK4, true>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, s32);
}

int batch2d_max_blocks_per_sm(bool mix) {
  int n = 0;
  const size_t sm = mix ? s2::smem_bytes<true, true>() : s2::smem_bytes<true, false>();
  if (mix)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage2d_batch<SMAUG_INT_RK4, true>, NTHREADS, sm);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage2d_batch<SMAUG_INT_RK4, false>, NTHREADS, sm);
  return n;
}

