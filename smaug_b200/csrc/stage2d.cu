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

// ---------------------------------------------------------------------------
// Fixed ghost layers of a 2D stage.  The reference's 2D gravity
// (grav_parallel, src/centdiff2.cu:721-787) and background energy coupling
// (src/centdiff2.cu:587-717) run on every cell with i < n0-2 and j < n1-2 --
// the two low ghost layers included -- and its driver (source_parallel,
// src/centdiff2.cu:790-872) on every cell; a fixed boundary never rewrites
// those ghost cells, so they evolve.  One thread per cell of the fixed
// layers (dim-0 layers first, then the dim-1 layers between them) applies
// those terms from the stage input, combines like the stage kernel, writes
// the cell and its images along the other (non-fixed) dimension, and adds
// their fast speeds to the stage's CFL maxima.  At a ghost cell the
// derivatives along the fixed dimension vanish (grad3dn covers [2, n-3]);
// along the other one they use the reference's velocities, which it
// computes only on cells with some coordinate in [2, n-3]
// (computevels_parallel strips, src/computedervfields.cu:18-126), 0 on the
// corner cells, and its edge zeroing (src/gradops.cu:459-474).
// ---------------------------------------------------------------------------
template <int MODE, bool MIX>
__global__ void __launch_bounds__(128) fixed_ghost2d_kernel(const KParams P, const KBufs B) {
  using ST = typename Form<MIX>::S;
  const ST* u = static_cast<const ST*>(B.uin);
  const int n0 = P.n0, n1 = P.n1;
  const long nc = P.ncell;
  const bool f0 = P.bc[0] == SMAUG_BC_FIXED, f1 = P.bc[1] == SMAUG_BC_FIXED;
  const int perA = f1 ? n1 : n1 - 4;
  const int lenA = f0 ? 4 * perA : 0;
  const int lenB = f1 ? 4 * (n0 - 4) : 0;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  double cm0 = 0.0, cm1 = 0.0;
  if (t < lenA + lenB) {
    int i, j, fixdim;
    if (t < lenA) {
      const int layer = t / perA, b = t % perA;
      i = layer < 2 ? layer : n0 - 4 + layer;
      j = f1 ? b : b + 2;
      fixdim = 0;
    } else {
      t -= lenA;
      const int layer = t / (n0 - 4), b = t % (n0 - 4);
      j = layer < 2 ? layer : n1 - 4 + layer;
      i = b + 2;
      fixdim = 1;
    }
    const double dt = *B.dt_new;
    const double tstage = B.stage == 0 ? *B.t_prev : *B.t_prev + (B.stage == 3 ? dt : 0.5 * dt);
    const long c = (long)j * n0 + i;
    double s[6];
#pragma unroll
    for (int f = 0; f < 6; f++) s[f] = (double)u[f * nc + c];
    const double eb = B.bg[0 * nc + c], rb = B.bg[1 * nc + c], bb[2] = {B.bg[2 * nc + c], B.bg[3 * nc + c]};
    double inc[6] = {0, 0, 0, 0, 0, 0};
    const bool lowok = i < n0 - 2 && j < n1 - 2;
    if (lowok && P.has_bg) {
      // velocity component comp at (ii, jj) as computevels leaves it
      auto vel = [&](int comp, int ii, int jj) -> double {
        if (!((ii >= 2 && ii <= n0 - 3) || (jj >= 2 && jj <= n1 - 3))) return 0.0;
        const long cc = (long)jj * n0 + ii;
        return (double)u[(1 + comp) * nc + cc] / ((double)u[cc] + B.bg[1 * nc + cc]);
      };
      // grad3dn of v_comp along dim a at (i, j)
      auto gv = [&](int comp, int a) -> double {
        const int x = a == 0 ? i : j, n = a == 0 ? n0 : n1;
        if (!(x > 1 && x < n - 2)) return 0.0;
        double w[5];
#pragma unroll
        for (int q = 0; q < 5; q++) w[q] = a == 0 ? vel(comp, i + q - 2, j) : vel(comp, i, j + q - 2);
        double g = d4(w, 2, 1, 0.5 / B.delx[a][x]);
        if (P.bt[a] != 0) {
          const int o = a == 0 ? j : i, no = a == 0 ? n1 : n0;
          const bool others = o >= 2 && o <= no - 3;
          if (x == n - 3 || (x == n - 4 && others) || x == 2 || (x == 3 && others)) g = 0.0;
        }
        return g;
      };
      const double ptb = (P.gamma - 1) * eb - 0.5 * (P.gamma - 2) * (bb[0] * bb[0] + bb[1] * bb[1]);
#pragma unroll
      for (int dir = 0; dir < 2; dir++) {
        inc[EN] -= dt * ptb * gv(dir, dir);
#pragma unroll
        for (int idim = 0; idim < 2; idim++) inc[EN] += dt * bb[idim] * bb[dir] * gv(dir, idim);
      }
    }
    if (lowok && P.has_grav) {
      inc[M1] += dt * P.g[0] * s[RHO];
      inc[M2] += dt * P.g[1] * s[RHO];
      const double rt = s[RHO] + rb;
      inc[EN] += (dt * s[RHO]) * (P.g[0] * s[M1]) / rt;
      inc[EN] += (dt * s[RHO]) * (P.g[1] * s[M2]) / rt;
    }
    if (P.driver == SMAUG_DRIVER_GAUSS) {
      double v = P.drv_amp;
      if (P.drv_period > 0) v *= sin(tstage * 2.0 * M_PI / P.drv_period);
      if (P.drv_sigma[0] > 0) {
        const double x = B.pos[0][i] - P.drv_x0[0];
        v *= exp(-x * x / (P.drv_sigma[0] * P.drv_sigma[0]));
      }
      if (P.drv_sigma[1] > 0) {
        const double x = B.pos[1][j] - P.drv_x0[1];
        v *= exp(-x * x / (P.drv_sigma[1] * P.drv_sigma[1]));
      }
      inc[M1] += dt * v * (s[RHO] + rb);
    }
    double res[6];
    const bool is_base = (MODE == SMAUG_INT_EULER) || B.stage == 3;
    if (MODE == SMAUG_INT_EULER) {
#pragma unroll
      for (int f = 0; f < 6; f++) res[f] = (MIX ? base_value<MIX>(B, f * nc + c) : s[f]) + inc[f];
    } else {
      const double wgt = (B.stage == 0 || B.stage == 3) ? 1.0 / 6.0 : 1.0 / 3.0;
      const double cst = (B.stage == 2) ? 1.0 : 0.5;
#pragma unroll
      for (int f = 0; f < 6; f++) {
        const double dl = inc[f];
        if (B.stage == 0) {
          const double u0 = MIX ? base_value<MIX>(B, f * nc + c) : s[f];
          B.acc[f * nc + c] = u0 + wgt * dl;
          res[f] = u0 + cst * dl;
        } else if (B.stage < 3) {
          B.acc[f * nc + c] = B.acc[f * nc + c] + wgt * dl;
          res[f] = base_value<MIX>(B, f * nc + c) + cst * dl;
        } else {
          res[f] = B.acc[f * nc + c] + wgt * dl;
        }
      }
    }
    bool bad = false;
#pragma unroll
    for (int f = 0; f < 6; f++) bad |= !isfinite(res[f]);
    if (bad) atomicOr(B.flags, 1);
    // the cell and its images along the other dimension (none when that
    // dimension is fixed too)
    const int od = 1 - fixdim;
    int img[3];
    img[0] = od == 0 ? i : j;
    const int nimg = 1 + ((od == 0 ? f0 : f1) ? 0 : ghost_images(img[0], od == 0 ? n0 : n1, P.bc[od], img + 1));
    bool negated = false;
    for (int q = 0; q < nimg; q++) {
      const long cc = od == 0 ? (long)j * n0 + img[q] : (long)img[q] * n0 + i;
      const bool neg = (q > 0) && P.gneg[od];
      if (neg != negated) {
#pragma unroll
        for (int f = 0; f < 6; f++) res[f] = -res[f];
        negated = neg;
      }
#pragma unroll
      for (int f = 0; f < 6; f++) store_value<MIX>(B, f * nc + cc, res[f], is_base);
      double c0, c1;
      cfast2_both(P.gamma, res[RHO], res[M1], res[M2], res[EN], res[B1], res[B2], B.bg[0 * nc + cc],
                  B.bg[1 * nc + cc], B.bg[2 * nc + cc], B.bg[3 * nc + cc], c0, c1);
      cm0 = dmax0(cm0, c0);
      cm1 = dmax0(cm1, c1);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    cm0 = dmax0(cm0, __shfl_xor_sync(0xffffffffu, cm0, o));
    cm1 = dmax0(cm1, __shfl_xor_sync(0xffffffffu, cm1, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&B.cmax_out[0], (unsigned long long)__double_as_longlong(cm0));
    atomicMax(&B.cmax_out[1], (unsigned long long)__double_as_longlong(cm1));
  }
}

cudaError_t launch_fixed_ghost2d(int mode, bool mix, const KParams& K, const KBufs& B, cudaStream_t st) {
  const bool f0 = K.bc[0] == SMAUG_BC_FIXED, f1 = K.bc[1] == SMAUG_BC_FIXED;
  const int n = (f0 ? 4 * (f1 ? K.n1 : K.n1 - 4) : 0) + (f1 ? 4 * (K.n0 - 4) : 0);
  if (n == 0) return cudaSuccess;
  const unsigned grid = (unsigned)((n + 127) / 128);
  if (mode == SMAUG_INT_EULER) {
    if (mix) fixed_ghost2d_kernel<SMAUG_INT_EULER, true><<<grid, 128, 0, st>>>(K, B);
    else fixed_ghost2d_kernel<SMAUG_INT_EULER, false><<<grid, 128, 0, st>>>(K, B);
  } else {
    if (mix) fixed_ghost2d_kernel<SMAUG_INT_RK4, true><<<grid, 128, 0, st>>>(K, B);
    else fixed_ghost2d_kernel<SMAUG_INT_RK4, false><<<grid, 128, 0, st>>>(K, B);
  }
  return cudaGetLastError();
}

cudaError_t stage2d_set_attributes() {
  cudaError_t e;
#define SMAUG_ATTR2(M, BG, MIX)                                              \
  if ((e = stage2d_attr<M, BG, MIX, false>())) return e;                   \
  if ((e = stage2d_attr<M, BG, MIX, true>())) return e;
  SMAUG_ATTR2(SMAUG_INT_EULER, true, false)
  SMAUG_ATTR2(SMAUG_INT_EULER, false, false)
  SMAUG_ATTR2(SMAUG_INT_RK4, true, false)
  SMAUG_ATTR2(SMAUG_INT_RK4, false, false)
  SMAUG_ATTR2(SMAUG_INT_EULER, true, true)
  SMAUG_ATTR2(SMAUG_INT_EULER, false, true)
  SMAUG_ATTR2(SMAUG_INT_RK4, true, true)
  SMAUG_ATTR2(SMAUG_INT_RK4, false, true)
#undef SMAUG_ATTR2
  return cudaSuccess;
}

}  // namespace smaug
