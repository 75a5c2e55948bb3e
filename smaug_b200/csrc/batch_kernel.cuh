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

// Grid barrier of the persistent kernel: every block arrives once per
// barrier and the last to arrive opens the next generation.  The wait is
// bounded (about 2^25 polls of 64 ns, a few seconds against a stage of about
// a millisecond): a block that gives up sets *err and the kernel ends, so a
// fault elsewhere cannot hang the GPU.  Returns false when the launch must
// stop.
__device__ __forceinline__ bool batch_grid_sync(BatchSync* s, int* err, unsigned nblocks) {
  __shared__ int stop;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    volatile unsigned int* gen = &s->gen;
    const unsigned int g = *gen;
    __threadfence();  // this block's writes of the stage before its arrival
    if (atomicAdd(&s->count, 1u) == nblocks - 1) {
      atomicExch(&s->count, 0u);
      __threadfence();
      atomicAdd(&s->gen, 1u);
    } else {
      long polls = 0;
      while (*gen == g) {
        if (++polls > (1L << 25)) {
          atomicOr(err, 1);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    stop = *(volatile int*)err;
  }
  __syncthreads();
  return stop == 0;
}

// Several RK4 steps (steps k0 .. k0+nsteps-1 of the batch, which fix each
// stage's buffer-block variant) of every run in one launch: in each stage the
// blocks take tiles from a shared counter, one at a time (taking four at a
// time unbalanced the ends of the stages: 4.98 against 4.76 ms per step for
// 64 runs), until the list is done, then meet at the grid barrier.  Launched cooperatively with at most as many blocks as fit
// on the GPU at once.  Stage inputs written by other blocks earlier in the
// launch are read through L2 (the CG form of the stage body).
template <bool MIX>
__global__ void __launch_bounds__(NTHREADS, SMAUG_MINB2D)
    stage2d_batch_cycle(const KParams* __restrict__ Ks, const KBufs* __restrict__ Bs,
                        const int4* __restrict__ tiles, int ntiles, int nruns, int k0, int nsteps,
                        BatchSync* sync, int* err) {
  __shared__ int tile_s;
  for (int k = k0; k < k0 + nsteps; k++) {
    const int parity = k % 2;
    for (int s = 0; s < 4; s++) {
      const int ring = (4 * k + s) % 3;
      const KBufs* Bv = Bs + (size_t)((s * 2 + parity) * 3 + ring) * nruns;
      int* ctr = &sync->next[(k - k0) * 4 + s];
      for (;;) {
        if (threadIdx.x == 0 && threadIdx.y == 0) tile_s = atomicAdd(ctr, 1);
        __syncthreads();
        const int it = tile_s;
        __syncthreads();
        if (it >= ntiles) break;
        const int4 t = tiles[it];  // run, tile x, tile y
        stage2d_body<SMAUG_INT_RK4, true, MIX, false, true>(Ks[t.x], Bv[t.x], t.y, t.z);
        __syncthreads();
      }
      if (!batch_grid_sync(sync, err, gridDim.x)) return;
    }
  }
}

cudaError_t launch_batch2d_cycle(bool mix, const KParams* Ks, const KBufs* Bs, const int4* tiles,
                                 int ntiles, int nruns, int k0, int nsteps, BatchSync* sync, int* err,
                                 int grid, cudaStream_t st) {
  if (nsteps < 1 || nsteps > BATCH_MAX_STEPS) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(sync, 0, sizeof(BatchSync), st);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(TX, TY);
  cfg.dynamicSmemBytes = mix ? s2::smem_bytes<true, true>() : s2::smem_bytes<true, false>();
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (mix)
    return cudaLaunchKernelEx(&cfg, stage2d_batch_cycle<true>, Ks, Bs, tiles, ntiles, nruns, k0, nsteps,
                              sync, err);
  return cudaLaunchKernelEx(&cfg, stage2d_batch_cycle<false>, Ks, Bs, tiles, ntiles, nruns, k0, nsteps,
                            sync, err);
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
  if ((e = cudaFuncSetAttribute(stage2d_batch_cycle<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64)))
    return e;
  if ((e = cudaFuncSetAttribute(stage2d_batch_cycle<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s32)))
    return e;
  return cudaFuncSetAttribute(stage2d_batch<SMAUG_INT_RK4, true>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, s32);
}

int batch2d_cycle_max_blocks_per_sm(bool mix) {
  int n = 0;
  const size_t sm = mix ? s2::smem_bytes<true, true>() : s2::smem_bytes<true, false>();
  if (mix)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage2d_batch_cycle<true>, NTHREADS, sm);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage2d_batch_cycle<false>, NTHREADS, sm);
  return n;
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

