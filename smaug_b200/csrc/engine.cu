// engine.cu -- B200 (sm_100a) time-advance engine for SMAUG, FP64.
//
// One fused kernel per stage evaluates the whole spatial operator of the
// reference's single-stage step (src/iosmaug.c:631-835) for a 2D tile
// (stage2d.cuh) or a 3D tile (stage3d.cuh):
//   state tile + 3-cell halo staged in shared memory
//   -> directional fluxes + 4th-order divergence     (src/centdiff1.cu, centdiff2.cu)
//   -> background energy coupling, gravity            (src/centdiff2.cu:80-154)
//   -> hyperdiffusion nu_r/nu_l and sources            (src/hyperdifvisc1{r,l}.cu,
//                                                      src/hyperdif*source*.cu)
//   -> user driver                                     (source_parallel)
//   -> stage combine (Euler or classical RK4), ghost images (src/boundary.cu)
//   -> per-dimension CFL maxima of the written state (src/computedervfields.cu:1864-2050)
// The CFL maxima of a stage's input are produced by the previous launch's
// epilogue, so no launch waits for the host: a step is 1 (Euler) or 4 (RK4)
// launches and the dt rule (src/iosmaug.c:541-616) runs on the device.
//
// Arithmetic follows the reference's expression trees term by term (same
// divisions, same accumulation order per cell) so that results agree with the
// reference's FP64 output to rounding.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/smaug_b200.h"
#include "engine_internal.h"
#include "kernels.cuh"

#define SMAUG_VERSION_STRING "smaug_b200 0.3 (sm_100a, fp64 + mixed, 2D+3D)"

namespace smaug {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

int set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}
void clear_error() { g_err.clear(); }
const char* last_error() { return g_err.c_str(); }

#define CUDA_TRY(call)                                                            \
  do {                                                                            \
    cudaError_t _e = (call);                                                      \
    if (_e != cudaSuccess)                                                        \
      return smaug::set_error(SMAUG_E_CUDA, "%s failed: %s (%s:%d)", #call,       \
                       cudaGetErrorString(_e), __FILE__, __LINE__);               \
  } while (0)

// ---------------------------------------------------------------------------
// auxiliary kernels: ghost fill and CFL maxima of an arbitrary state
// ---------------------------------------------------------------------------
__global__ void ghost_fill2d_kernel(const KParams P, double* u) {
  long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (c >= P.ncell) return;
  int i = (int)(c % P.n0), j = (int)(c / P.n0);
  int si = ghost_source(i, P.n0, P.bc[0]);
  int sj = ghost_source(j, P.n1, P.bc[1]);
  if (si == i && sj == j) return;
  long s = (long)sj * P.n0 + si;
  const bool neg = ((si != i) && P.gneg[0]) != ((sj != j) && P.gneg[1]);
  for (int f = 0; f < 6; f++) u[f * P.ncell + c] = neg ? -u[f * P.ncell + s] : u[f * P.ncell + s];
}

__global__ void ghost_fill3d_kernel(const KParams P, double* u) {
  long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (c >= P.ncell) return;
  int i = (int)(c % P.n0), j = (int)((c / P.n0) % P.n1), k = (int)(c / ((long)P.n0 * P.n1));
  int si = ghost_source(i, P.n0, P.bc[0]);
  int sj = ghost_source(j, P.n1, P.bc[1]);
  int sk = ghost_source(k, P.n2, P.bc[2]);
  if (si == i && sj == j && sk == k) return;
  long s = ((long)sk * P.n1 + sj) * P.n0 + si;
  const bool neg = (((si != i) && P.gneg[0]) != ((sj != j) && P.gneg[1])) != ((sk != k) && P.gneg[2]);
  for (int f = 0; f < 8; f++) u[f * P.ncell + c] = neg ? -u[f * P.ncell + s] : u[f * P.ncell + s];
}

// cells that the stage kernels never write: a ghost coordinate along a dim
// with fixed boundaries
__device__ __forceinline__ bool fixed_ghost(const KParams& P, int i, int j, int k) {
  return (P.bc[0] == SMAUG_BC_FIXED && (i < 2 || i > P.n0 - 3)) ||
         (P.bc[1] == SMAUG_BC_FIXED && (j < 2 || j > P.n1 - 3)) ||
         (P.n2 > 1 && P.bc[2] == SMAUG_BC_FIXED && (k < 2 || k > P.n2 - 3));
}

__global__ void cmax3d_kernel(const KParams P, const double* u, const double* bg,
                              unsigned long long* out, int fixed_only) {
  long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double cm[3] = {0, 0, 0};
  bool use = c < P.ncell;
  if (use && fixed_only)
    use = fixed_ghost(P, (int)(c % P.n0), (int)((c / P.n0) % P.n1), (int)(c / ((long)P.n0 * P.n1)));
  if (use) {
    const long nc = P.ncell;
    double s[8], g[5];
    for (int f = 0; f < 8; f++) s[f] = u[f * nc + c];
    for (int f = 0; f < 5; f++) g[f] = bg[f * nc + c];
    cfast3_all(P.gamma, s, g, cm);
  }
  for (int d = 0; d < 3; d++) {
    double v = cm[d];
    if (!(v > 0)) v = 0.0;
    for (int o = 16; o > 0; o >>= 1) v = dmax0(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&out[d], (unsigned long long)__double_as_longlong(v));
  }
}

__global__ void cmax2d_kernel(const KParams P, const double* u, const double* bg,
                              unsigned long long* out, int fixed_only) {
  long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double cm[2] = {0, 0};
  bool use = c < P.ncell;
  if (use && fixed_only) use = fixed_ghost(P, (int)(c % P.n0), (int)(c / P.n0), 0);
  if (use) {
    const long nc = P.ncell;
    cfast2_both(P.gamma, u[0 * nc + c], u[1 * nc + c], u[2 * nc + c], u[3 * nc + c], u[4 * nc + c],
                u[5 * nc + c], bg[0 * nc + c], bg[1 * nc + c], bg[2 * nc + c], bg[3 * nc + c], cm[0],
                cm[1]);
  }
  for (int d = 0; d < 2; d++) {
    double v = cm[d];
    if (!(v > 0)) v = 0.0;
    for (int o = 16; o > 0; o >>= 1) v = dmax0(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&out[d], (unsigned long long)__double_as_longlong(v));
  }
}

// ---------------------------------------------------------------------------
// host engine
// ---------------------------------------------------------------------------
// One pending asynchronous .out write: the state is copied on the engine's
// stream into a pinned host buffer, and a host thread writes the file once the
// copy's event has completed.
struct Snapshot {
  double* host = nullptr;        // pinned, nvar * ncell doubles (allocated on first use)
  cudaEvent_t ready = nullptr;   // recorded after the device-to-host copies
  std::thread worker;
  int rc = SMAUG_OK;             // result of the write, read after the join
  std::string err;
};

struct Engine {
  smaug_params_t P{};
  KParams K{};
  int nd = 2, nevo = 6, nbg = 4;
  long ncell = 0;
  cudaStream_t stream = nullptr;
  bool mix = false;                      // mixed precision form
  double* d_u[3] = {nullptr, nullptr, nullptr};  // FP64 form: rotating state buffers
  float* d_h[4] = {nullptr, nullptr, nullptr, nullptr};  // mixed form: float buffers
  double* d_x64 = nullptr;               // mixed form: FP64 state for host copies
  double* d_acc = nullptr;
  double* d_bg = nullptr;
  double* d_delx[3] = {nullptr, nullptr, nullptr};
  double* d_pos[3] = {nullptr, nullptr, nullptr};
  int* d_pad[3] = {nullptr, nullptr, nullptr};
  unsigned long long* d_cmax = nullptr;  // ring of 3 x [3]
  double* d_dt = nullptr;                // [2]
  double* d_t = nullptr;                 // [2]
  int* d_flags = nullptr;
  std::vector<double> pos_host;          // positions after the metric rewrite
  int cur = 0;                           // buffer holding the current state
  long stage_count = 0;                  // launches so far (cmax ring position)
  int parity = 0;                        // dt/t double buffer
  int64_t it = 0;
  int device = 0;
  bool ghost_upd = false;                // 2D fixed ghost layers updated every stage
  bool tma_ok = false;                   // 2D: tensor maps of every stage input exist
  int tma = 0;                           // 2D staging: 0 per-thread loads, 1 bulk tensor copies
                                         // (persistent grid), 2 bulk tensor copies (a block per tile)
  TmaMap tm_u[3], tm_h[4], tm_bg;        // tensor maps of d_u / d_h / d_bg
  cudaStream_t own_stream = nullptr;     // created by the engine
  Snapshot snap[2];                      // asynchronous .out writes, used in turn
  int snap_next = 0;
  int snap_rc = SMAUG_OK;                // first failed write since the last wait
  std::string snap_err;
};

// wait for the write of slot s (if any) and keep its error
static void join_snapshot(Engine* e, Snapshot& s) {
  if (!s.worker.joinable()) return;
  s.worker.join();
  if (s.rc != SMAUG_OK && e->snap_rc == SMAUG_OK) {
    e->snap_rc = s.rc;
    e->snap_err = s.err;
  }
  s.rc = SMAUG_OK;
}

static void free_engine(Engine* e) {
  if (!e) return;
  for (Snapshot& s : e->snap) {
    join_snapshot(e, s);
    if (s.host) cudaFreeHost(s.host);
    if (s.ready) cudaEventDestroy(s.ready);
  }
  for (int i = 0; i < 3; i++) {
    cudaFree(e->d_u[i]);
    cudaFree(e->d_h[i]);
    cudaFree(e->d_delx[i]);
    cudaFree(e->d_pos[i]);
    cudaFree(e->d_pad[i]);
  }
  cudaFree(e->d_h[3]);
  cudaFree(e->d_x64);
  cudaFree(e->d_acc);
  cudaFree(e->d_bg);
  cudaFree(e->d_cmax);
  cudaFree(e->d_dt);
  cudaFree(e->d_t);
  cudaFree(e->d_flags);
  if (e->own_stream) cudaStreamDestroy(e->own_stream);
  delete e;
}

static int validate(const smaug_params_t* p) {
  if (!p) return set_error(SMAUG_E_INVALID, "null parameter block");
  if (p->version != SMAUG_PARAMS_VERSION)
    return set_error(SMAUG_E_INVALID, "parameter block version %d, expected %d", p->version,
                     SMAUG_PARAMS_VERSION);
  if (p->ndim != 2 && p->ndim != 3) return set_error(SMAUG_E_INVALID, "ndim must be 2 or 3 (got %d)", p->ndim);
  for (int d = 0; d < p->ndim; d++)
    if (p->n[d] < 8) return set_error(SMAUG_E_INVALID, "n[%d]=%d: need at least 4 interior cells", d, p->n[d]);
  {
    long long cells = 1;
    for (int d = 0; d < p->ndim; d++) cells *= p->n[d];
    if (cells >= (1LL << 31) - 2)
      return set_error(SMAUG_E_UNSUPPORTED, "%lld cells: grids are limited to 2^31-2 cells", cells);
  }
  if (p->integrator != SMAUG_INT_EULER && p->integrator != SMAUG_INT_RK4)
    return set_error(SMAUG_E_INVALID, "unknown integrator %d", p->integrator);
  if (p->precision != SMAUG_PREC_FP64 && p->precision != SMAUG_PREC_MIXED)
    return set_error(SMAUG_E_INVALID, "unknown precision form %d", p->precision);
  if (p->pad_model != SMAUG_PAD_STRAY && p->pad_model != SMAUG_PAD_ZERO)
    return set_error(SMAUG_E_INVALID, "unknown pad model %d", p->pad_model);
  for (int d = 0; d < p->ndim; d++) {
    int b = p->boundtype[d][0];
    if (b != p->boundtype[d][1])
      return set_error(SMAUG_E_UNSUPPORTED, "dim %d: different upper/lower boundary types", d);
    if (b != SMAUG_BC_PERIODIC && b != SMAUG_BC_CONTCD4 && b != SMAUG_BC_CONT && b != SMAUG_BC_SYMM &&
        b != SMAUG_BC_ASYMM && b != SMAUG_BC_FIXED)
      return set_error(SMAUG_E_UNSUPPORTED, "dim %d: boundary type %d not supported", d, b);
    // the reference adds the driver term to every cell, ghosts included
    // (src/centdiff2.cu:790-872), and fixed ghost cells keep it; the 2D
    // engine updates its fixed ghost layers as the reference does
    // (fixed_ghost2d_kernel), the 3D one does not
    if (b == SMAUG_BC_FIXED && p->driver != SMAUG_DRIVER_NONE && p->ndim == 3)
      return set_error(SMAUG_E_UNSUPPORTED, "dim %d: 3D fixed boundaries with a driver term", d);
  }
  if (p->moddton == 1 && !(p->courant > 0))
    return set_error(SMAUG_E_INVALID, "courant must be > 0 with moddton");
  if (!(p->gamma > 1.0)) return set_error(SMAUG_E_INVALID, "gamma must be > 1");
  if (p->driver != SMAUG_DRIVER_NONE && p->driver != SMAUG_DRIVER_GAUSS &&
      p->driver != SMAUG_DRIVER_GAUSS_STEP)
    return set_error(SMAUG_E_INVALID, "unknown driver %d", p->driver);
  if (p->stencil_order != 0 && p->stencil_order != 4 && p->stencil_order != 6)
    return set_error(SMAUG_E_INVALID, "stencil_order must be 4 or 6 (got %d)", p->stencil_order);
  return SMAUG_OK;
}

// Source cells of the stray tmp6 stores that land in the right pad along
// each dim (src/hyperdifvisc1r.cu:1235,1255): the store of cell t goes to
// linear index t + off of the padded array (off = n0+1 in 2D,
// n0*n1+n0+1 in 3D); the pad cell of transverse row r along dim d is
// padded (n_d+1) with the other coordinates +1.
static std::vector<int> pad_sources(const smaug_params_t* p, int dim) {
  int nd = p->ndim;
  long n[3] = {p->n[0], p->n[1], nd == 3 ? p->n[2] : 1};
  long m[3] = {n[0] + 2, n[1] + 2, nd == 3 ? n[2] + 2 : 1};
  long dimp = n[0] * n[1] * n[2];
  long off = (nd == 3) ? n[0] * n[1] + n[0] + 1 : n[0] + 1;
  std::vector<int> src;
  if (nd == 2) {
    int o = 1 - dim;
    src.assign(n[o], -1);
    for (long r = 0; r < n[o]; r++) {
      long P0 = (dim == 0) ? n[0] + 1 : r + 1;
      long P1 = (dim == 0) ? r + 1 : n[1] + 1;
      long L = P1 * m[0] + P0;
      long t = L - off;
      if (p->pad_model == SMAUG_PAD_STRAY && t >= 0 && t < dimp) src[r] = (int)t;
    }
  } else {
    // across index: the two other coordinates, lower axis fastest
    int a1 = dim == 0 ? 1 : 0, a2 = dim == 2 ? 1 : 2;
    src.assign(n[a1] * n[a2], -1);
    for (long v = 0; v < n[a2]; v++)
      for (long u = 0; u < n[a1]; u++) {
        long P[3];
        P[dim] = n[dim] + 1;
        P[a1] = u + 1;
        P[a2] = v + 1;
        long L = (P[2] * m[1] + P[1]) * m[0] + P[0];
        long t = L - off;
        if (p->pad_model == SMAUG_PAD_STRAY && t >= 0 && t < dimp) src[v * n[a1] + u] = (int)t;
      }
  }
  return src;
}

static int create(const smaug_params_t* p, const double* w, const double* pos, Engine** out) {
  int rc = validate(p);
  if (rc) return rc;
  if (!w || !pos || !out) return set_error(SMAUG_E_INVALID, "null array argument");
  Engine* e = new Engine();
  e->P = *p;
  e->nd = p->ndim;
  e->nevo = 2 + 2 * e->nd;
  e->nbg = 2 + e->nd;
  e->ncell = 1;
  for (int d = 0; d < e->nd; d++) e->ncell *= p->n[d];
  const long nc = e->ncell;
  const int nvar = 4 + 3 * e->nd;
  // grid metric on the host (initgrid), then 1D metric arrays
  e->pos_host.assign(pos, pos + (size_t)e->nd * nc);
  std::vector<double> delx((size_t)e->nd * nc);
  grid_metric(e->nd, p->n, e->pos_host.data(), delx.data());
  std::vector<double> dl1[3], ps1[3];
  const int n2 = (e->nd == 3) ? p->n[2] : 1;
  for (int d = 0; d < e->nd; d++) {
    dl1[d].assign(p->n[d], 0.0);
    ps1[d].assign(p->n[d], 0.0);
    // representative interior line; every interior cell must agree
    for (int a = 0; a < p->n[d]; a++) {
      int ijk[3] = {2, 2, e->nd == 3 ? 2 : 0};
      ijk[d] = a;
      long c = ((long)ijk[2] * p->n[1] + ijk[1]) * p->n[0] + ijk[0];
      dl1[d][a] = delx[(size_t)d * nc + c];
      ps1[d][a] = e->pos_host[(size_t)d * nc + c];
    }
    const int klo = (e->nd == 3) ? 2 : 0, khi = (e->nd == 3) ? n2 - 3 : 0;
    for (int k = klo; k <= khi; k++)
      for (int j = 2; j <= p->n[1] - 3; j++)
        for (int i = 2; i <= p->n[0] - 3; i++) {
          long c = ((long)k * p->n[1] + j) * p->n[0] + i;
          int a = (d == 0) ? i : (d == 1 ? j : k);
          if (delx[(size_t)d * nc + c] != dl1[d][a] ||
              (p->driver != SMAUG_DRIVER_NONE && e->pos_host[(size_t)d * nc + c] != ps1[d][a])) {
            delete e;
            return set_error(SMAUG_E_UNSUPPORTED,
                             "grid metric along dim %d varies across lines (cell %d,%d,%d); only "
                             "tensor-product grids are supported", d, i, j, k);
          }
          if (!(dl1[d][a] > 0)) {
            delete e;
            return set_error(SMAUG_E_INVALID, "non-positive cell width along dim %d at %d", d, a);
          }
        }
  }
  // kernel parameters
  KParams& K = e->K;
  K.n0 = p->n[0];
  K.n1 = p->n[1];
  K.n2 = n2;
  K.ncell = nc;
  set_boundaries(K, p, e->nd);
  K.order6 = p->stencil_order == 6;
  for (int d = 0; d < 3; d++) {
    K.dx[d] = p->dx[d];
    K.g[d] = p->g[d];
    K.drv_x0[d] = p->drv_x0[d];
    K.drv_sigma[d] = p->drv_sigma[d];
  }
  K.gamma = p->gamma;
  K.courant = p->courant;
  K.dtmax = p->dtmax;
  for (int f = 0; f < SMAUG_MAXVAR; f++) K.chyp[f] = p->chyp[f];
  K.moddton = p->moddton;
  K.hyperdif = p->hyperdifmom;
  K.has_grav = 0;
  for (int d = 0; d < e->nd; d++) if (p->g[d] != 0.0) K.has_grav = 1;
  K.has_bg = 0;
  for (int f = 2 + 2 * e->nd; f < nvar && !K.has_bg; f++)
    for (long c = 0; c < nc; c++)
      if (w[(size_t)f * nc + c] != 0.0) { K.has_bg = 1; break; }
  // The reference's 2D gravity (src/centdiff2.cu:721-787), background
  // energy coupling (src/centdiff2.cu:587-717) and driver (every cell) also
  // update ghost cells, and fixed boundaries never overwrite them there: the
  // fixed ghost layers drift.  fixed_ghost2d_kernel reproduces that after
  // every 2D stage; the 3D kernels stay interior and 3D fixed boundaries with
  // these terms match the reference (its 3D kernels are bounded to the
  // interior).
  e->ghost_upd = e->nd == 2 && has_fixed(K) && (K.has_bg || K.has_grav || p->driver != SMAUG_DRIVER_NONE);
  if (e->ghost_upd && p->stencil_order == 6) {
    delete e;
    return set_error(SMAUG_E_UNSUPPORTED,
                     "2D fixed boundaries with gravity, background fields or a driver use the "
                     "4th-order stencil");
  }
  K.driver = p->driver;
  K.drv_amp = p->drv_amp;
  K.drv_period = p->drv_period;
  // device buffers
  int dev = 0;
  cudaGetDevice(&dev);
  e->device = dev;
  auto fail = [&](int code) { free_engine(e); return code; };
#define E_TRY(call)                                                                             \
  do {                                                                                          \
    cudaError_t _e = (call);                                                                    \
    if (_e != cudaSuccess)                                                                      \
      return fail(set_error(_e == cudaErrorMemoryAllocation ? SMAUG_E_NOMEM : SMAUG_E_CUDA,    \
                            "%s: %s", #call, cudaGetErrorString(_e)));                         \
  } while (0)
  E_TRY(cudaStreamCreateWithFlags(&e->own_stream, cudaStreamNonBlocking));
  e->stream = e->own_stream;
  size_t evo_bytes = sizeof(double) * e->nevo * nc;
  e->mix = (p->precision == SMAUG_PREC_MIXED);
  if (e->mix) {
    for (int i = 0; i < 4; i++) E_TRY(cudaMalloc(&e->d_h[i], sizeof(float) * e->nevo * nc));
    E_TRY(cudaMalloc(&e->d_x64, evo_bytes));
  } else {
    for (int i = 0; i < 3; i++) E_TRY(cudaMalloc(&e->d_u[i], evo_bytes));
  }
  if (p->integrator == SMAUG_INT_RK4) E_TRY(cudaMalloc(&e->d_acc, evo_bytes));
  E_TRY(cudaMalloc(&e->d_bg, sizeof(double) * e->nbg * nc));
  for (int d = 0; d < e->nd; d++) {
    E_TRY(cudaMalloc(&e->d_delx[d], sizeof(double) * p->n[d]));
    E_TRY(cudaMalloc(&e->d_pos[d], sizeof(double) * p->n[d]));
    E_TRY(cudaMemcpy(e->d_delx[d], dl1[d].data(), sizeof(double) * p->n[d], cudaMemcpyHostToDevice));
    E_TRY(cudaMemcpy(e->d_pos[d], ps1[d].data(), sizeof(double) * p->n[d], cudaMemcpyHostToDevice));
    std::vector<int> ps = pad_sources(p, d);
    E_TRY(cudaMalloc(&e->d_pad[d], sizeof(int) * ps.size()));
    E_TRY(cudaMemcpy(e->d_pad[d], ps.data(), sizeof(int) * ps.size(), cudaMemcpyHostToDevice));
  }
  E_TRY(cudaMalloc(&e->d_cmax, sizeof(unsigned long long) * 12));  // ring of 3 + fixed floor
  E_TRY(cudaMalloc(&e->d_dt, sizeof(double) * 2));
  E_TRY(cudaMalloc(&e->d_t, sizeof(double) * 2));
  E_TRY(cudaMalloc(&e->d_flags, sizeof(int)));
  E_TRY(cudaMemcpy(e->mix ? e->d_x64 : e->d_u[0], w, evo_bytes, cudaMemcpyHostToDevice));
  E_TRY(cudaMemcpy(e->d_bg, w + (size_t)e->nevo * nc, sizeof(double) * e->nbg * nc,
                   cudaMemcpyHostToDevice));
  double dt0[2] = {p->dt, p->dt}, t0[2] = {0.0, 0.0};
  E_TRY(cudaMemcpy(e->d_dt, dt0, sizeof(dt0), cudaMemcpyHostToDevice));
  E_TRY(cudaMemcpy(e->d_t, t0, sizeof(t0), cudaMemcpyHostToDevice));
  E_TRY(cudaMemset(e->d_flags, 0, sizeof(int)));
  E_TRY(stage2d_set_attributes());
  E_TRY(stage3d_set_attributes());
  // 2D: tensor maps for the bulk tensor staging when the grid admits it
  // (selected by smaug_set_staging; per-thread loads by default)
  if (e->nd == 2 && stage2d_tma_supported(e->K, e->mix)) {
    E_TRY(stage2d_tma_set_attributes());
    bool ok = true;
    for (int i = 0; i < 3 && ok; i++)
      if (e->d_u[i]) ok = stage2d_tma_encode(&e->tm_u[i], e->d_u[i], false, e->K, e->nevo, e->nevo) == 0;
    for (int i = 0; i < 4 && ok; i++)
      if (e->d_h[i]) ok = stage2d_tma_encode(&e->tm_h[i], e->d_h[i], true, e->K, e->nevo, e->nevo) == 0;
    if (ok) ok = stage2d_tma_encode(&e->tm_bg, e->d_bg, false, e->K, e->nbg, e->K.has_bg ? 4 : 1) == 0;
    e->tma_ok = ok;
    e->tma = 0;
  }
#undef E_TRY
  *out = e;
  return SMAUG_OK;
}

// tensor map of an engine buffer that is a stage input (null if none)
static const TmaMap* tma_map_of(const Engine* e, const void* uin) {
  for (int i = 0; i < 3; i++)
    if (e->d_u[i] && uin == e->d_u[i]) return &e->tm_u[i];
  for (int i = 0; i < 4; i++)
    if (e->d_h[i] && uin == e->d_h[i]) return &e->tm_h[i];
  return nullptr;
}

// FP64 state of the host interface <-> float high/low pair of the mixed form
__global__ void split_kernel(const double* x, float* hi, float* lo, long n) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = x[i];
  const float h = (float)v;
  hi[i] = h;
  lo[i] = (float)(v - (double)h);
}
__global__ void join_kernel(const float* hi, const float* lo, double* x, long n) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = (double)hi[i] + (double)lo[i];
}

// the float pair holding the current base state (mixed form)
static float* base_hi(Engine* e) { return e->d_h[2 * e->cur]; }
static float* base_lo(Engine* e) { return e->d_h[2 * e->cur + 1]; }

// FP64 view of the current state: the state itself (FP64 form) or the
// conversion buffer filled from the high/low pair (mixed form)
static int current_fp64(Engine* e, double** out) {
  if (!e->mix) {
    *out = e->d_u[e->cur];
    return SMAUG_OK;
  }
  const long n = (long)e->nevo * e->ncell;
  join_kernel<<<(unsigned)((n + 255) / 256), 256, 0, e->stream>>>(base_hi(e), base_lo(e), e->d_x64, n);
  CUDA_TRY(cudaGetLastError());
  *out = e->d_x64;
  return SMAUG_OK;
}

// ghost fill of the state just set (the FP64 buffer) + CFL maxima into the
// ring slot of the next launch; the mixed form then splits it into its pair
static int reset_derived(Engine* e) {
  const int bs = 256;
  long nb = (e->ncell + bs - 1) / bs;
  double* u = e->mix ? e->d_x64 : e->d_u[e->cur];
  if (e->nd == 3)
    ghost_fill3d_kernel<<<(unsigned)nb, bs, 0, e->stream>>>(e->K, u);
  else
    ghost_fill2d_kernel<<<(unsigned)nb, bs, 0, e->stream>>>(e->K, u);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemsetAsync(e->d_cmax, 0, sizeof(unsigned long long) * 9, e->stream));
  unsigned long long* slot = e->d_cmax + 3 * (e->stage_count % 3);
  if (e->nd == 3)
    cmax3d_kernel<<<(unsigned)nb, bs, 0, e->stream>>>(e->K, u, e->d_bg, slot, 0);
  else
    cmax2d_kernel<<<(unsigned)nb, bs, 0, e->stream>>>(e->K, u, e->d_bg, slot, 0);
  CUDA_TRY(cudaGetLastError());
  const long n = (long)e->nevo * e->ncell;
  if (e->mix) {
    split_kernel<<<(unsigned)((n + bs - 1) / bs), bs, 0, e->stream>>>(u, base_hi(e), base_lo(e), n);
    CUDA_TRY(cudaGetLastError());
  }
  if (has_fixed(e->K)) {
    // fixed ghost cells are written by no stage: every buffer gets them now,
    // and their CFL maxima become the floor of every later maximum
    if (!e->mix) {
      for (int i = 0; i < 3; i++)
        if (e->d_u[i] && e->d_u[i] != u)
          CUDA_TRY(cudaMemcpyAsync(e->d_u[i], u, sizeof(double) * n, cudaMemcpyDeviceToDevice, e->stream));
    } else {
      const int other = 1 - e->cur;
      split_kernel<<<(unsigned)((n + bs - 1) / bs), bs, 0, e->stream>>>(u, e->d_h[2 * other],
                                                                          e->d_h[2 * other + 1], n);
      CUDA_TRY(cudaGetLastError());
      if (e->P.integrator == SMAUG_INT_RK4)  // h2, h3 are plain stage buffers
        CUDA_TRY(cudaMemcpyAsync(e->d_h[3], e->d_h[2], sizeof(float) * n, cudaMemcpyDeviceToDevice,
                                 e->stream));
    }
    if (e->ghost_upd) {
      // the fixed ghost layers change: fixed_ghost2d_kernel adds their CFL
      // speeds to every stage's maxima, so there is no constant floor
      for (int d = 0; d < 3; d++) e->K.cmax_floor[d] = 0.0;
      return SMAUG_OK;
    }
    unsigned long long* fl = e->d_cmax + 9;
    CUDA_TRY(cudaMemsetAsync(fl, 0, sizeof(unsigned long long) * 3, e->stream));
    if (e->nd == 3)
      cmax3d_kernel<<<(unsigned)nb, bs, 0, e->stream>>>(e->K, u, e->d_bg, fl, 1);
    else
      cmax2d_kernel<<<(unsigned)nb, bs, 0, e->stream>>>(e->K, u, e->d_bg, fl, 1);
    CUDA_TRY(cudaGetLastError());
    double floor3[3] = {0, 0, 0};
    CUDA_TRY(cudaMemcpyAsync(floor3, fl, sizeof(floor3), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (int d = 0; d < 3; d++) e->K.cmax_floor[d] = d < e->nd ? floor3[d] : 0.0;
  }
  return SMAUG_OK;
}

// kernel buffer block of one stage launch; uin/un/uout are the FP64 buffers
// or the float buffers of the mixed form (un_lo / uout_lo: low parts where a
// base state is read or written); `ring` = the launch's CFL-maxima ring slot
// (stage_count mod 3), `parity` = the step's dt/t double-buffer index
static KBufs fill_kbufs(const Engine* e, int mode, int stage, int parity, int ring, const void* uin,
                        const void* un, const float* un_lo, void* uout, float* uout_lo) {
  KBufs B{};
  B.uin = uin;
  B.un = un;
  B.un_lo = un_lo;
  B.uout = uout;
  B.uout_lo = uout_lo;
  B.acc = e->d_acc;
  B.bg = e->d_bg;
  for (int d = 0; d < 3; d++) {
    B.delx[d] = e->d_delx[d];
    B.pos[d] = e->d_pos[d];
    B.padsrc[d] = e->d_pad[d];
  }
  B.cmax_in = reinterpret_cast<const double*>(e->d_cmax + 3 * ring);
  B.cmax_out = e->d_cmax + 3 * ((ring + 1) % 3);
  B.cmax_clear = e->d_cmax + 3 * ((ring + 2) % 3);
  B.dt_prev = e->d_dt + parity;
  B.dt_new = e->d_dt + (1 - parity);
  B.t_prev = e->d_t + parity;
  B.t_new = e->d_t + (1 - parity);
  B.flags = e->d_flags;
  B.mode = mode;
  B.stage = stage;
  return B;
}

static int launch_stage(Engine* e, int mode, int stage, const void* uin, const void* un,
                        const float* un_lo, void* uout, float* uout_lo) {
  KBufs B = fill_kbufs(e, mode, stage, e->parity, (int)(e->stage_count % 3), uin, un, un_lo, uout,
                       uout_lo);
  // a driver that acts in one step only: the kernels see the plain Gaussian
  // driver in that step and none in the others
  KParams K = e->K;
  if (K.driver == SMAUG_DRIVER_GAUSS_STEP)
    K.driver = (e->it == e->P.drv_step) ? SMAUG_DRIVER_GAUSS : SMAUG_DRIVER_NONE;
  if (e->nd == 3) {
    CUDA_TRY(launch_stage3d_any(mode, e->mix, K, B, e->stream));
  } else {
    const TmaMap* ms = e->tma ? tma_map_of(e, uin) : nullptr;
    if (ms)
      CUDA_TRY(launch_stage2d_tma(mode, e->mix, K, B, *ms, e->tm_bg, e->tma == 1, e->stream));
    else
      CUDA_TRY(launch_stage2d_any(mode, e->mix, K, B, e->stream));
    if (e->ghost_upd) CUDA_TRY(launch_fixed_ghost2d(mode, e->mix, K, B, e->stream));
  }
  e->stage_count++;
  return SMAUG_OK;
}

// RK4 stage buffers of an engine: (uin, un, un_lo, uout, uout_lo) of stage s;
// the base state stays in place for RK4 (FP64: d_u[cur]; mixed: h0/h1)
static KBufs rk4_kbufs(const Engine* e, int stage, int parity, int ring) {
  if (e->mix) {
    float* hi = e->d_h[0];
    float* lo = e->d_h[1];
    switch (stage) {
      case 0: return fill_kbufs(e, SMAUG_INT_RK4, 0, parity, ring, hi, hi, lo, e->d_h[2], nullptr);
      case 1: return fill_kbufs(e, SMAUG_INT_RK4, 1, parity, ring, e->d_h[2], hi, lo, e->d_h[3], nullptr);
      case 2: return fill_kbufs(e, SMAUG_INT_RK4, 2, parity, ring, e->d_h[3], hi, lo, e->d_h[2], nullptr);
      default: return fill_kbufs(e, SMAUG_INT_RK4, 3, parity, ring, e->d_h[2], hi, lo, hi, lo);
    }
  }
  double* un = e->d_u[e->cur];
  double* a = e->d_u[(e->cur + 1) % 3];
  double* b = e->d_u[(e->cur + 2) % 3];
  switch (stage) {
    case 0: return fill_kbufs(e, SMAUG_INT_RK4, 0, parity, ring, un, un, nullptr, a, nullptr);
    case 1: return fill_kbufs(e, SMAUG_INT_RK4, 1, parity, ring, a, un, nullptr, b, nullptr);
    case 2: return fill_kbufs(e, SMAUG_INT_RK4, 2, parity, ring, b, un, nullptr, a, nullptr);
    default: return fill_kbufs(e, SMAUG_INT_RK4, 3, parity, ring, a, un, nullptr, un, nullptr);
  }
}

static int sync_check(Engine* e) {
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  int flags = 0;
  CUDA_TRY(cudaMemcpy(&flags, e->d_flags, sizeof(int), cudaMemcpyDeviceToHost));
  if (flags & FLAG_TMA_TIMEOUT) {
    CUDA_TRY(cudaMemset(e->d_flags, 0, sizeof(int)));
    return set_error(SMAUG_E_CUDA, "a bulk tensor copy of a stage tile did not complete in time (by step %lld)",
                     (long long)e->it);
  }
  if (flags & 1) {
    CUDA_TRY(cudaMemset(e->d_flags, 0, sizeof(int)));
    return set_error(SMAUG_E_NONFINITE, "non-finite value in the evolved state by step %lld",
                     (long long)e->it);
  }
  return SMAUG_OK;
}

static int enqueue_steps(Engine* e, int nsteps) {
  for (int s = 0; s < nsteps; s++) {
    int rc;
    if (e->mix) {
      if (e->P.integrator == SMAUG_INT_EULER) {
        // base-state pairs (h0,h1) and (h2,h3) alternate
        int nxt = 1 - e->cur;
        rc = launch_stage(e, SMAUG_INT_EULER, 0, base_hi(e), base_hi(e), base_lo(e),
                          e->d_h[2 * nxt], e->d_h[2 * nxt + 1]);
        if (rc) return rc;
        e->cur = nxt;
      } else {
        // base state in (h0,h1); stage states in h2, h3
        float* hi = e->d_h[0];
        float* lo = e->d_h[1];
        if ((rc = launch_stage(e, SMAUG_INT_RK4, 0, hi, hi, lo, e->d_h[2], nullptr))) return rc;
        if ((rc = launch_stage(e, SMAUG_INT_RK4, 1, e->d_h[2], hi, lo, e->d_h[3], nullptr))) return rc;
        if ((rc = launch_stage(e, SMAUG_INT_RK4, 2, e->d_h[3], hi, lo, e->d_h[2], nullptr))) return rc;
        if ((rc = launch_stage(e, SMAUG_INT_RK4, 3, e->d_h[2], hi, lo, hi, lo))) return rc;
      }
    } else if (e->P.integrator == SMAUG_INT_EULER) {
      int nxt = (e->cur + 1) % 3;
      rc = launch_stage(e, SMAUG_INT_EULER, 0, e->d_u[e->cur], e->d_u[e->cur], nullptr,
                        e->d_u[nxt], nullptr);
      if (rc) return rc;
      e->cur = nxt;
    } else {
      int a = (e->cur + 1) % 3, b = (e->cur + 2) % 3;
      double* un = e->d_u[e->cur];
      if ((rc = launch_stage(e, SMAUG_INT_RK4, 0, un, un, nullptr, e->d_u[a], nullptr))) return rc;
      if ((rc = launch_stage(e, SMAUG_INT_RK4, 1, e->d_u[a], un, nullptr, e->d_u[b], nullptr))) return rc;
      if ((rc = launch_stage(e, SMAUG_INT_RK4, 2, e->d_u[b], un, nullptr, e->d_u[a], nullptr))) return rc;
      if ((rc = launch_stage(e, SMAUG_INT_RK4, 3, e->d_u[a], un, nullptr, un, nullptr))) return rc;
    }
    e->parity = 1 - e->parity;
    e->it++;
  }
  return SMAUG_OK;
}

static int step(Engine* e, int nsteps) {
  int rc = enqueue_steps(e, nsteps);
  if (rc) return rc;
  return sync_check(e);
}

}  // namespace smaug

// ===========================================================================
// C ABI
// ===========================================================================
using smaug::Engine;

extern "C" const char* smaug_last_error(void) { return smaug::last_error(); }
extern "C" const char* smaug_version(void) { return SMAUG_VERSION_STRING; }

extern "C" int smaug_params_default(smaug_params_t* p, int32_t ndim) {
  smaug::clear_error();
  if (!p || (ndim != 2 && ndim != 3)) return smaug::set_error(SMAUG_E_INVALID, "bad arguments");
  memset(p, 0, sizeof(*p));
  p->version = SMAUG_PARAMS_VERSION;
  p->ndim = ndim;
  p->n[0] = p->n[1] = 132;
  p->n[2] = (ndim == 3) ? 132 : 1;
  p->moddton = 1;
  p->hyperdifmom = 1;
  p->integrator = SMAUG_INT_EULER;
  p->precision = SMAUG_PREC_FP64;
  p->pad_model = SMAUG_PAD_STRAY;
  for (int d = 0; d < 3; d++) p->dx[d] = (d < ndim) ? 2.0 * M_PI / 128.0 : 0.0;
  p->dt = 1.0e-8;
  p->dtmax = 1.0;
  p->courant = 0.3;
  p->gamma = 5.0 / 3.0;
  for (int f = 0; f < SMAUG_MAXVAR; f++) p->chyp[f] = 0.2;
  return SMAUG_OK;
}

extern "C" int smaug_create(const smaug_params_t* p, const double* w, const double* pos,
                            smaug_handle_t* out) {
  smaug::clear_error();
  if (!out) return smaug::set_error(SMAUG_E_INVALID, "null handle pointer");
  *out = nullptr;
  Engine* e = nullptr;
  int rc = smaug::create(p, w, pos, &e);
  if (rc) return rc;
  rc = smaug::reset_derived(e);
  if (!rc) {
    cudaError_t ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) rc = smaug::set_error(SMAUG_E_CUDA, "create: %s", cudaGetErrorString(ce));
  }
  if (rc) {
    smaug::free_engine(e);
    return rc;
  }
  *out = reinterpret_cast<smaug_handle_t>(e);
  return SMAUG_OK;
}

static Engine* H(smaug_handle_t h) { return reinterpret_cast<Engine*>(h); }

extern "C" int smaug_step(smaug_handle_t h, int32_t nsteps) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  if (nsteps < 0) return smaug::set_error(SMAUG_E_INVALID, "nsteps < 0");
  return smaug::step(H(h), nsteps);
}

extern "C" int smaug_step_async(smaug_handle_t h, int32_t nsteps) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  if (nsteps < 0) return smaug::set_error(SMAUG_E_INVALID, "nsteps < 0");
  return smaug::enqueue_steps(H(h), nsteps);
}

extern "C" int smaug_sync(smaug_handle_t h) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  return smaug::sync_check(H(h));
}

extern "C" int smaug_set_stream(smaug_handle_t h, void* stream) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  Engine* e = H(h);
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  e->stream = stream ? static_cast<cudaStream_t>(stream) : e->own_stream;
  return SMAUG_OK;
}

extern "C" int smaug_get_state(smaug_handle_t h, double* w) {
  smaug::clear_error();
  if (!h || !w) return smaug::set_error(SMAUG_E_INVALID, "null argument");
  Engine* e = H(h);
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  double* u = nullptr;
  int rc = smaug::current_fp64(e, &u);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(w, u, sizeof(double) * e->nevo * e->ncell, cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  CUDA_TRY(cudaMemcpy(w + (size_t)e->nevo * e->ncell, e->d_bg, sizeof(double) * e->nbg * e->ncell,
                      cudaMemcpyDeviceToHost));
  return SMAUG_OK;
}

extern "C" int smaug_get_fields(smaug_handle_t h, double* w, int32_t f0, int32_t nf) {
  smaug::clear_error();
  if (!h || !w) return smaug::set_error(SMAUG_E_INVALID, "null argument");
  Engine* e = H(h);
  const int nvar = e->nevo + e->nbg;
  if (f0 < 0 || nf < 0 || f0 + nf > nvar)
    return smaug::set_error(SMAUG_E_INVALID, "fields [%d, %d) outside [0, %d)", f0, f0 + nf, nvar);
  if (nf == 0) return SMAUG_OK;
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  const size_t nc = (size_t)e->ncell;
  const int fe = f0 + nf < e->nevo ? f0 + nf : e->nevo;  // end of the evolved part
  if (f0 < e->nevo) {
    double* u = nullptr;
    int rc = smaug::current_fp64(e, &u);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(w, u + (size_t)f0 * nc, sizeof(double) * (fe - f0) * nc,
                             cudaMemcpyDeviceToHost, e->stream));
  }
  const int b0 = f0 > e->nevo ? f0 : e->nevo;
  if (f0 + nf > e->nevo)
    CUDA_TRY(cudaMemcpyAsync(w + (size_t)(b0 - f0) * nc, e->d_bg + (size_t)(b0 - e->nevo) * nc,
                             sizeof(double) * (f0 + nf - b0) * nc, cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return SMAUG_OK;
}

extern "C" int smaug_set_state(smaug_handle_t h, const double* w) {
  smaug::clear_error();
  if (!h || !w) return smaug::set_error(SMAUG_E_INVALID, "null argument");
  Engine* e = H(h);
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  CUDA_TRY(cudaMemcpyAsync(e->mix ? e->d_x64 : e->d_u[e->cur], w, sizeof(double) * e->nevo * e->ncell,
                           cudaMemcpyHostToDevice, e->stream));
  int rc = smaug::reset_derived(e);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return SMAUG_OK;
}

extern "C" int smaug_get_time(smaug_handle_t h, int64_t* it, double* t, double* dt) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  Engine* e = H(h);
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  double tb[2], db[2];
  CUDA_TRY(cudaMemcpy(tb, e->d_t, sizeof(tb), cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(db, e->d_dt, sizeof(db), cudaMemcpyDeviceToHost));
  if (it) *it = e->it;
  if (t) *t = tb[e->parity];
  if (dt) *dt = db[e->parity];
  return SMAUG_OK;
}

extern "C" int smaug_get_cmax(smaug_handle_t h, double* cmax) {
  smaug::clear_error();
  if (!h || !cmax) return smaug::set_error(SMAUG_E_INVALID, "null argument");
  Engine* e = H(h);
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  double c[3];
  CUDA_TRY(cudaMemcpy(c, e->d_cmax + 3 * (e->stage_count % 3), sizeof(c), cudaMemcpyDeviceToHost));
  for (int d = 0; d < e->nd; d++) cmax[d] = c[d];
  return SMAUG_OK;
}

extern "C" int smaug_staging(smaug_handle_t h, int32_t* tma, int32_t* available) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  Engine* e = H(h);
  if (tma) *tma = e->tma;
  if (available) *available = e->tma_ok ? 1 : 0;
  return SMAUG_OK;
}

extern "C" int smaug_set_staging(smaug_handle_t h, int32_t tma) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  Engine* e = H(h);
  if (tma < 0 || tma > 2) return smaug::set_error(SMAUG_E_INVALID, "staging %d not in {0, 1, 2}", tma);
  if (tma && !e->tma_ok)
    return smaug::set_error(SMAUG_E_UNSUPPORTED,
                            "bulk tensor staging needs a 2D grid whose rows are a multiple of 16 bytes "
                            "in the storage type and the 4th-order stencil");
  e->tma = tma;
  return SMAUG_OK;
}

extern "C" int smaug_write_out(smaug_handle_t h, const char* path, const char* name, int32_t it,
                               double t) {
  smaug::clear_error();
  if (!h || !path) return smaug::set_error(SMAUG_E_INVALID, "null argument");
  Engine* e = H(h);
  std::vector<double> w((size_t)(e->nevo + e->nbg) * e->ncell);
  int rc = smaug_get_state(h, w.data());
  if (rc) return rc;
  return smaug::write_out_host(path, &e->P, w.data(), e->pos_host.data(), name, it, t);
}

// Asynchronous .out snapshot: enqueue the copies on the engine's stream and
// return; a host thread writes the file when they complete.  Two slots are
// used in turn, so a third call waits for the write of the first.
extern "C" int smaug_write_out_async(smaug_handle_t h, const char* path, const char* name, int32_t it,
                                     double t) {
  smaug::clear_error();
  if (!h || !path) return smaug::set_error(SMAUG_E_INVALID, "null argument");
  Engine* e = H(h);
  smaug::Snapshot& s = e->snap[e->snap_next];
  smaug::join_snapshot(e, s);
  const size_t nc = (size_t)e->ncell;
  const size_t nvar = (size_t)(e->nevo + e->nbg);
  if (!s.host) {
    if (cudaMallocHost(&s.host, sizeof(double) * nvar * nc) != cudaSuccess) {
      cudaGetLastError();
      s.host = nullptr;
      return smaug::set_error(SMAUG_E_NOMEM, "pinned snapshot buffer of %zu bytes", sizeof(double) * nvar * nc);
    }
  }
  if (!s.ready) CUDA_TRY(cudaEventCreateWithFlags(&s.ready, cudaEventDisableTiming));
  double* u = nullptr;
  int rc = smaug::current_fp64(e, &u);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(s.host, u, sizeof(double) * e->nevo * nc, cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaMemcpyAsync(s.host + (size_t)e->nevo * nc, e->d_bg, sizeof(double) * e->nbg * nc,
                           cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaEventRecord(s.ready, e->stream));
  std::string spath(path), sname(name ? name : "");
  const smaug_params_t P = e->P;
  const double* pos = e->pos_host.data();
  smaug::Snapshot* sp = &s;
  s.worker = std::thread([sp, spath, sname, P, pos, it, t]() {
    if (cudaEventSynchronize(sp->ready) != cudaSuccess) {
      sp->rc = SMAUG_E_CUDA;
      sp->err = std::string("snapshot copy: ") + cudaGetErrorString(cudaGetLastError());
      return;
    }
    sp->rc = smaug::write_out_host(spath.c_str(), &P, sp->host, pos, sname.c_str(), it, t);
    if (sp->rc != SMAUG_OK) sp->err = smaug::last_error();
  });
  e->snap_next ^= 1;
  return SMAUG_OK;
}

extern "C" int smaug_wait_writes(smaug_handle_t h) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null argument");
  Engine* e = H(h);
  for (smaug::Snapshot& s : e->snap) smaug::join_snapshot(e, s);
  const int rc = e->snap_rc;
  e->snap_rc = SMAUG_OK;
  if (rc != SMAUG_OK) return smaug::set_error(rc, "%s", e->snap_err.c_str());
  return SMAUG_OK;
}

extern "C" int smaug_destroy(smaug_handle_t h) {
  smaug::clear_error();
  if (!h) return SMAUG_OK;
  Engine* e = H(h);
  cudaStreamSynchronize(e->stream);
  smaug::free_engine(e);
  return SMAUG_OK;
}

// ===========================================================================
// Batched ensemble of 2D runs
// ===========================================================================
// Independent runs advance together over the concatenated tile list of all
// runs, in one of two forms the autotuner chooses between: one launch of
// stage2d_batch per stage, or one persistent launch of stage2d_batch_cycle
// for several steps (its blocks meet at a grid barrier between stages).  A
// cycle of 6 RK4 steps (the period of the dt/t double buffers, 2, and of the
// CFL-maxima ring, 3 slots advanced 4 times per step) is captured once into a
// CUDA graph and replayed: 24 stage launches, or one persistent launch.  Each
// run keeps its own engine state (buffers, dt, time, CFL maxima), so a run's
// results are those of the same run stepped alone.
namespace smaug {

constexpr int BATCH_CYCLE = 6;

// tile shapes of the batched kernel, each its own instantiation
struct BatchShape {
  int tx, ty;
  cudaError_t (*launch)(int, bool, const KParams*, const KBufs*, const int4*, int, int, cudaStream_t);
  cudaError_t (*launch_cycle)(bool, const KParams*, const KBufs*, const int4*, int, int, int, int, BatchSync*,
                              int*, int, cudaStream_t);
  cudaError_t (*set_attributes)();
  int (*max_blocks_per_sm)(bool);
  int (*cycle_max_blocks_per_sm)(bool);
};
constexpr int NSHAPES = 2;
static const BatchShape kShapes[NSHAPES] = {
    {32, 8, t32x8::launch_batch2d, t32x8::launch_batch2d_cycle, t32x8::batch2d_set_attributes,
     t32x8::batch2d_max_blocks_per_sm, t32x8::batch2d_cycle_max_blocks_per_sm},
    {16, 16, t16x16::launch_batch2d, t16x16::launch_batch2d_cycle, t16x16::batch2d_set_attributes,
     t16x16::batch2d_max_blocks_per_sm, t16x16::batch2d_cycle_max_blocks_per_sm},
};
// candidates per tile shape: 4 grids of per-stage launches, then the
// persistent launch
constexpr int NCAND = 5;

struct Batch {
  std::vector<Engine*> runs;
  bool mix = false;
  cudaStream_t stream = nullptr;
  KParams* d_K = nullptr;   // [nruns]
  KBufs* d_B = nullptr;     // [4 stages][2 parities][3 ring slots][nruns]
  int4* d_tiles[NSHAPES] = {nullptr, nullptr};  // (run, tile x, tile y) per tile shape
  int ntiles[NSHAPES] = {0, 0};
  int shape = 0;            // tile shape in use (index into kShapes)
  int pinned = -1;          // tile shape fixed by the caller (-1: tuned)
  int grid = 0;             // persistent blocks per launch (0: not chosen yet)
  int grid_candidates[NSHAPES][4] = {};
  float grid_ms[NSHAPES][4] = {};
  int tuned = 0;            // (shape, grid) candidates timed so far
  bool persistent = false;  // the chosen form: the persistent launch
  int pin_form = -1;        // -1 tuned, 0 per-stage launches only, 1 persistent only
  int cycle_grid[NSHAPES] = {};   // blocks of the persistent launch (all co-resident)
  float cycle_ms[NSHAPES] = {};   // its step time per tile shape
  BatchSync* d_sync = nullptr;    // its grid barrier and tile counters
  int* d_err = nullptr;           // set when one of its barrier waits gave up
  long steps = 0;
  cudaGraphExec_t cycle = nullptr;
  cudaStream_t own_stream = nullptr;  // the batch's stream while a caller stream is set
};

static void free_batch(Batch* b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->cycle) cudaGraphExecDestroy(b->cycle);
  cudaFree(b->d_K);
  cudaFree(b->d_B);
  cudaFree(b->d_sync);
  cudaFree(b->d_err);
  for (int s = 0; s < NSHAPES; s++) cudaFree(b->d_tiles[s]);
  for (Engine* e : b->runs) free_engine(e);
  cudaStreamDestroy(b->own_stream ? b->own_stream : b->stream);
  delete b;
}

static int batch_variant(int stage, int parity, int ring) { return (stage * 2 + parity) * 3 + ring; }

// one RK4 step of every run, starting at global step index k of the batch,
// with tile shape `shape` and `grid` persistent blocks
static int batch_enqueue_step(Batch* b, long k, int shape, int grid) {
  const int nr = (int)b->runs.size();
  const int parity = (int)(k % 2);
  for (int s = 0; s < 4; s++) {
    const int ring = (int)((4 * k + s) % 3);
    CUDA_TRY(kShapes[shape].launch(SMAUG_INT_RK4, b->mix, b->d_K,
                                   b->d_B + (size_t)batch_variant(s, parity, ring) * nr, b->d_tiles[shape],
                                   b->ntiles[shape], grid, b->stream));
  }
  return SMAUG_OK;
}

// nsteps (<= BATCH_MAX_STEPS) RK4 steps of every run from global step k in one
// persistent launch with tile shape `shape`
static int batch_enqueue_persistent(Batch* b, long k, int nsteps, int shape) {
  CUDA_TRY(kShapes[shape].launch_cycle(b->mix, b->d_K, b->d_B, b->d_tiles[shape], b->ntiles[shape],
                                       (int)b->runs.size(), (int)(k % BATCH_CYCLE), nsteps, b->d_sync,
                                       b->d_err, b->cycle_grid[shape], b->stream));
  return SMAUG_OK;
}

static void batch_advance_bookkeeping(Batch* b, long nsteps) {
  for (Engine* e : b->runs) {
    e->stage_count += 4 * nsteps;
    if (nsteps % 2) e->parity = 1 - e->parity;
    e->it += nsteps;
  }
  b->steps += nsteps;
}

static int batch_create(int nruns, const smaug_params_t* const* params, const double* const* w,
                        const double* const* pos, Batch** out) {
  if (nruns < 1 || !params || !w || !pos || !out) return set_error(SMAUG_E_INVALID, "bad batch arguments");
  Batch* b = new Batch();
  auto fail = [&](int code) { free_batch(b); return code; };
  for (int r = 0; r < nruns; r++) {
    if (!params[r]) return fail(set_error(SMAUG_E_INVALID, "run %d: null parameter block", r));
    if (params[r]->ndim != 2) return fail(set_error(SMAUG_E_UNSUPPORTED, "run %d: batches are 2D only", r));
    if (params[r]->integrator != SMAUG_INT_RK4)
      return fail(set_error(SMAUG_E_UNSUPPORTED, "run %d: batches step with RK4", r));
    if (params[r]->precision != params[0]->precision)
      return fail(set_error(SMAUG_E_UNSUPPORTED, "run %d: all runs of a batch share one precision form", r));
    if (params[r]->stencil_order == 6)
      return fail(set_error(SMAUG_E_UNSUPPORTED, "run %d: batches use the 4th-order stencil", r));
    if (params[r]->driver == SMAUG_DRIVER_GAUSS_STEP)
      return fail(set_error(SMAUG_E_UNSUPPORTED, "run %d: batches replay steps; a one-step driver "
                                                 "is not supported", r));
    Engine* e = nullptr;
    int rc = create(params[r], w[r], pos[r], &e);
    if (rc) return fail(rc);
    b->runs.push_back(e);
    if (e->ghost_upd)
      return fail(set_error(SMAUG_E_UNSUPPORTED, "run %d: batches keep fixed ghost layers constant; "
                                                 "gravity, background fields or a driver update them", r));
    rc = reset_derived(e);
    if (rc) return fail(rc);
  }
  b->mix = (params[0]->precision == SMAUG_PREC_MIXED);
  cudaError_t ce = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (ce != cudaSuccess) return fail(set_error(SMAUG_E_CUDA, "stream: %s", cudaGetErrorString(ce)));
  for (Engine* e : b->runs) {
    ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) return fail(set_error(SMAUG_E_CUDA, "create: %s", cudaGetErrorString(ce)));
    e->stream = b->stream;
  }
  // parameter blocks, the 24 buffer-block variants of every run, the tile list
  std::vector<KParams> K(nruns);
  std::vector<KBufs> B((size_t)24 * nruns);
  std::vector<int4> tiles[NSHAPES];
  for (int r = 0; r < nruns; r++) {
    Engine* e = b->runs[r];
    K[r] = e->K;
    K[r].has_bg = 1;
    for (int s = 0; s < 4; s++)
      for (int par = 0; par < 2; par++)
        for (int ring = 0; ring < 3; ring++)
          B[(size_t)batch_variant(s, par, ring) * nruns + r] = rk4_kbufs(e, s, par, ring);
    for (int sh = 0; sh < NSHAPES; sh++) {
      const int sx = kShapes[sh].tx, sy = kShapes[sh].ty;
      const int tx = (e->K.n0 - 4 + sx - 1) / sx, ty = (e->K.n1 - 4 + sy - 1) / sy;
      for (int j = 0; j < ty; j++)
        for (int i = 0; i < tx; i++) tiles[sh].push_back(make_int4(r, i, j, 0));
    }
  }
#define B_TRY(call)                                                                             \
  do {                                                                                          \
    cudaError_t _e = (call);                                                                    \
    if (_e != cudaSuccess)                                                                      \
      return fail(set_error(_e == cudaErrorMemoryAllocation ? SMAUG_E_NOMEM : SMAUG_E_CUDA,    \
                            "%s: %s", #call, cudaGetErrorString(_e)));                         \
  } while (0)
  B_TRY(cudaMalloc(&b->d_K, sizeof(KParams) * nruns));
  B_TRY(cudaMalloc(&b->d_B, sizeof(KBufs) * B.size()));
  B_TRY(cudaMemcpy(b->d_K, K.data(), sizeof(KParams) * nruns, cudaMemcpyHostToDevice));
  B_TRY(cudaMemcpy(b->d_B, B.data(), sizeof(KBufs) * B.size(), cudaMemcpyHostToDevice));
  int dev = 0, nsm = 0;
  B_TRY(cudaGetDevice(&dev));
  B_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  for (int sh = 0; sh < NSHAPES; sh++) {
    const int nt = (int)tiles[sh].size();
    b->ntiles[sh] = nt;
    B_TRY(cudaMalloc(&b->d_tiles[sh], sizeof(int4) * nt));
    B_TRY(cudaMemcpy(b->d_tiles[sh], tiles[sh].data(), sizeof(int4) * nt, cudaMemcpyHostToDevice));
    B_TRY(kShapes[sh].set_attributes());
    // launch-shape candidates: 1, 2 or the occupancy limit of blocks per SM
    // (persistent), or one block per tile
    int occ = kShapes[sh].max_blocks_per_sm(b->mix);
    if (occ < 1) occ = 1;
    int* gc = b->grid_candidates[sh];
    gc[0] = nsm < nt ? nsm : nt;
    gc[1] = 2 * nsm < nt ? 2 * nsm : nt;
    gc[2] = occ * nsm < nt ? occ * nsm : nt;
    gc[3] = nt;
    // the persistent launch: every block resident at once
    int occ_c = kShapes[sh].cycle_max_blocks_per_sm(b->mix);
    b->cycle_grid[sh] = occ_c >= 1 ? (occ_c * nsm < nt ? occ_c * nsm : nt) : 0;
  }
  B_TRY(cudaMalloc(&b->d_sync, sizeof(BatchSync)));
  B_TRY(cudaMalloc(&b->d_err, sizeof(int)));
  B_TRY(cudaMemset(b->d_err, 0, sizeof(int)));
#undef B_TRY
  *out = b;
  return SMAUG_OK;
}

// Tile- and launch-shape autotuning: the first steps run with every
// (tile shape, grid) candidate -- 2 tile shapes x 4 grids, or the 4 grids of
// a pinned shape -- each timed with events; the fastest is kept.  Neither
// choice changes a cell's arithmetic (the tile only decides which block
// stages and computes it), so results do not depend on them.
// the two timing events of batch_tune, destroyed on every exit path
struct EventPair {
  cudaEvent_t ev[2] = {nullptr, nullptr};
  ~EventPair() {
    for (cudaEvent_t& e : ev)
      if (e) cudaEventDestroy(e);
  }
};

static int batch_tune(Batch* b, int* nsteps) {
  EventPair pair;
  cudaEvent_t* ev = pair.ev;
  CUDA_TRY(cudaEventCreate(&ev[0]));
  CUDA_TRY(cudaEventCreate(&ev[1]));
  auto wanted = [&](int sh, int g) {
    if (b->pinned >= 0 && sh != b->pinned) return false;
    if (g == NCAND - 1) return b->pin_form != 0 && b->cycle_grid[sh] > 0;
    return b->pin_form != 1;
  };
  for (int c = b->tuned; c < NSHAPES * NCAND && *nsteps > 0; c++) {
    const int sh = c / NCAND, g = c % NCAND;
    b->tuned = c + 1;
    if (!wanted(sh, g)) continue;
    CUDA_TRY(cudaEventRecord(ev[0], b->stream));
    int rc = g == NCAND - 1 ? batch_enqueue_persistent(b, b->steps, 1, sh)
                            : batch_enqueue_step(b, b->steps, sh, b->grid_candidates[sh][g]);
    if (rc) return rc;
    CUDA_TRY(cudaEventRecord(ev[1], b->stream));
    CUDA_TRY(cudaEventSynchronize(ev[1]));
    CUDA_TRY(cudaEventElapsedTime(g == NCAND - 1 ? &b->cycle_ms[sh] : &b->grid_ms[sh][g], ev[0], ev[1]));
    batch_advance_bookkeeping(b, 1);
    (*nsteps)--;
  }
  if (b->tuned == NSHAPES * NCAND) {
    int bs = -1, bg = 0;
    float best = 0;
    for (int sh = 0; sh < NSHAPES; sh++)
      for (int g = 0; g < NCAND; g++) {
        if (!wanted(sh, g)) continue;
        const float ms = g == NCAND - 1 ? b->cycle_ms[sh] : b->grid_ms[sh][g];
        if (bs < 0 || ms < best) bs = sh, bg = g, best = ms;
      }
    if (bs < 0) return set_error(SMAUG_E_CUDA, "no launch form of the batch could be timed");
    b->shape = bs;
    b->persistent = bg == NCAND - 1;
    b->grid = b->persistent ? b->cycle_grid[bs] : b->grid_candidates[bs][bg];
  }
  return SMAUG_OK;
}

static int batch_enqueue(Batch* b, int nsteps) {
  if (!b->grid) {
    int rc = batch_tune(b, &nsteps);
    if (rc) return rc;
  }
  while (nsteps > 0) {
    if (b->steps % BATCH_CYCLE == 0 && nsteps >= BATCH_CYCLE) {
      if (!b->cycle) {
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int rc = SMAUG_OK;
        if (b->persistent)
          rc = batch_enqueue_persistent(b, 0, BATCH_CYCLE, b->shape);
        else
          for (int k = 0; k < BATCH_CYCLE && !rc; k++) rc = batch_enqueue_step(b, k, b->shape, b->grid);
        cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (rc || ce != cudaSuccess) {
          if (g) cudaGraphDestroy(g);
          if (rc) return rc;
          return set_error(SMAUG_E_CUDA, "graph capture: %s", cudaGetErrorString(ce));
        }
        ce = cudaGraphInstantiate(&b->cycle, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return set_error(SMAUG_E_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
      }
      CUDA_TRY(cudaGraphLaunch(b->cycle, b->stream));
      batch_advance_bookkeeping(b, BATCH_CYCLE);
      nsteps -= BATCH_CYCLE;
    } else {
      int rc = b->persistent ? batch_enqueue_persistent(b, b->steps, 1, b->shape)
                             : batch_enqueue_step(b, b->steps, b->shape, b->grid);
      if (rc) return rc;
      batch_advance_bookkeeping(b, 1);
      nsteps--;
    }
  }
  return SMAUG_OK;
}

static int batch_sync(Batch* b) {
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  int err = 0;
  CUDA_TRY(cudaMemcpy(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) return set_error(SMAUG_E_CUDA, "persistent batch launch: a grid-barrier wait timed out");
  for (Engine* e : b->runs) {
    int rc = sync_check(e);
    if (rc) return rc;
  }
  return SMAUG_OK;
}

}  // namespace smaug

using smaug::Batch;
static Batch* HB(smaug_batch_t h) { return reinterpret_cast<Batch*>(h); }

extern "C" int smaug_batch_create(int32_t nruns, const smaug_params_t* const* params,
                                  const double* const* w, const double* const* pos,
                                  smaug_batch_t* out) {
  smaug::clear_error();
  if (!out) return smaug::set_error(SMAUG_E_INVALID, "null handle pointer");
  *out = nullptr;
  Batch* b = nullptr;
  int rc = smaug::batch_create(nruns, params, w, pos, &b);
  if (rc) return rc;
  *out = reinterpret_cast<smaug_batch_t>(b);
  return SMAUG_OK;
}

extern "C" int smaug_batch_step(smaug_batch_t h, int32_t nsteps) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  if (nsteps < 0) return smaug::set_error(SMAUG_E_INVALID, "nsteps < 0");
  int rc = smaug::batch_enqueue(HB(h), nsteps);
  if (rc) return rc;
  return smaug::batch_sync(HB(h));
}

extern "C" int smaug_batch_step_async(smaug_batch_t h, int32_t nsteps) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  if (nsteps < 0) return smaug::set_error(SMAUG_E_INVALID, "nsteps < 0");
  return smaug::batch_enqueue(HB(h), nsteps);
}

extern "C" int smaug_batch_sync(smaug_batch_t h) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  return smaug::batch_sync(HB(h));
}

extern "C" int smaug_batch_set_stream(smaug_batch_t h, void* stream) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  Batch* b = HB(h);
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  if (!b->own_stream) b->own_stream = b->stream;
  b->stream = stream ? static_cast<cudaStream_t>(stream) : b->own_stream;
  for (smaug::Engine* e : b->runs) e->stream = b->stream;
  return SMAUG_OK;
}

extern "C" int smaug_batch_get_state(smaug_batch_t h, int32_t run, double* w) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  Batch* b = HB(h);
  if (run < 0 || run >= (int)b->runs.size()) return smaug::set_error(SMAUG_E_INVALID, "run %d out of range", run);
  return smaug_get_state(reinterpret_cast<smaug_handle_t>(b->runs[run]), w);
}

extern "C" int smaug_batch_get_time(smaug_batch_t h, int32_t run, int64_t* it, double* t, double* dt) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  Batch* b = HB(h);
  if (run < 0 || run >= (int)b->runs.size()) return smaug::set_error(SMAUG_E_INVALID, "run %d out of range", run);
  return smaug_get_time(reinterpret_cast<smaug_handle_t>(b->runs[run]), it, t, dt);
}

extern "C" int smaug_batch_launch_shape(smaug_batch_t h, int32_t* grid, int32_t* candidates, float* ms) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  Batch* b = HB(h);
  if (grid) *grid = b->grid;
  for (int c = 0; c < 4; c++) {
    if (candidates) candidates[c] = b->grid_candidates[b->shape][c];
    if (ms) ms[c] = b->grid_ms[b->shape][c];
  }
  return SMAUG_OK;
}

extern "C" int smaug_batch_tile_shape(smaug_batch_t h, int32_t* tx, int32_t* ty, float* ms) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  Batch* b = HB(h);
  const bool chosen = b->grid != 0;
  if (tx) *tx = chosen ? smaug::kShapes[b->shape].tx : 0;
  if (ty) *ty = chosen ? smaug::kShapes[b->shape].ty : 0;
  if (ms)
    for (int sh = 0; sh < smaug::NSHAPES; sh++)
      for (int g = 0; g < 4; g++) ms[sh * 4 + g] = b->grid_ms[sh][g];
  return SMAUG_OK;
}

extern "C" int smaug_batch_persistent(smaug_batch_t h, int32_t* on, int32_t* grid, float* ms) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  Batch* b = HB(h);
  if (on) *on = b->grid != 0 && b->persistent ? 1 : 0;
  for (int sh = 0; sh < smaug::NSHAPES; sh++) {
    if (grid) grid[sh] = b->cycle_grid[sh];
    if (ms) ms[sh] = b->cycle_ms[sh];
  }
  return SMAUG_OK;
}

extern "C" int smaug_batch_pin_form(smaug_batch_t h, int32_t form) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  Batch* b = HB(h);
  if (b->tuned > 0 || b->grid != 0)
    return smaug::set_error(SMAUG_E_INVALID, "the launch form is chosen at the first step: pin it before");
  if (form < -1 || form > 1) return smaug::set_error(SMAUG_E_INVALID, "form must be -1, 0 or 1");
  if (form == 1)
    for (int sh = 0; sh < smaug::NSHAPES; sh++)
      if (b->cycle_grid[sh] <= 0 && (b->pinned < 0 || b->pinned == sh))
        return smaug::set_error(SMAUG_E_UNSUPPORTED, "no resident grid for the persistent launch");
  b->pin_form = form;
  return SMAUG_OK;
}

extern "C" int smaug_batch_pin_tile_shape(smaug_batch_t h, int32_t tx, int32_t ty) {
  smaug::clear_error();
  if (!h) return smaug::set_error(SMAUG_E_INVALID, "null handle");
  Batch* b = HB(h);
  if (b->tuned > 0 || b->grid != 0)
    return smaug::set_error(SMAUG_E_INVALID, "the tile shape is chosen at the first step: pin it before");
  for (int sh = 0; sh < smaug::NSHAPES; sh++)
    if (smaug::kShapes[sh].tx == tx && smaug::kShapes[sh].ty == ty) {
      b->pinned = sh;
      b->shape = sh;
      return SMAUG_OK;
    }
  return smaug::set_error(SMAUG_E_INVALID, "tile shape %dx%d not built (32x8, 16x16)", tx, ty);
}

extern "C" int smaug_batch_destroy(smaug_batch_t h) {
  smaug::clear_error();
  if (!h) return SMAUG_OK;
  smaug::free_batch(HB(h));
  return SMAUG_OK;
}

// ===========================================================================
// Allocation-free Euler step
// ===========================================================================
// Some callers cannot call cudaMalloc: applications that reserve their device
// memory up front (a framework's caching pool, a fixed per-process budget on
// a shared GPU) and refuse or cannot satisfy allocations made behind their
// back, plugins whose host forbids allocation inside its step callback, and
// loops that run beside other streams, where cudaFree's implicit device-wide
// synchronisation would stall them.  smaug_euler_step_noalloc serves them:
// the caller passes device buffers for the input and output state, and every
// piece of scratch the step needs (CFL maxima, dt and time words, the error
// flag, the 1D metric and the stray-pad source table) lives in the
// file-scope array below.
namespace smaug {

// Largest grid (cells per dimension, ghosts included) the array serves.
constexpr int NOALLOC_MAXN = 8192;
constexpr size_t NA_CMAX = 0;                                        // 9 x u64
constexpr size_t NA_DT = 128;                                        // 2 doubles
constexpr size_t NA_T = 160;                                         // 2 doubles
constexpr size_t NA_FLAGS = 192;                                     // 1 int
constexpr size_t NA_DELX = 256;                                      // 2 x MAXN doubles
constexpr size_t NA_PAD = NA_DELX + 2 * NOALLOC_MAXN * sizeof(double);  // 2 x MAXN ints
constexpr size_t NOALLOC_SCRATCH_BYTES = NA_PAD + 2 * NOALLOC_MAXN * sizeof(int);  // 196,864 B

// One copy per GPU that loads the library, held until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch per device (the host-side symbol is a
// stand-in, not a device address); looked up once, on a device's first call,
// and kept for the life of the process (a cudaDeviceReset invalidates it).
constexpr int NA_MAXDEV = 64;
static unsigned char* g_na_ptr[NA_MAXDEV] = {nullptr};
static std::mutex g_na_mu;

static int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAXDEV) return set_error(SMAUG_E_UNSUPPORTED, "device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return set_error(SMAUG_E_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch): %s", cudaGetErrorString(e));
    g_na_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_na_ptr[dev];
  return SMAUG_OK;
}

// stray-pad source cells (same rule as pad_sources on the host) into scratch
__global__ void noalloc_pad_kernel(int n0, int n1, int stray, int* pad0, int* pad1) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  long dimp = (long)n0 * n1, off = n0 + 1;
  if (r < n1) {  // dim 0: padded (n0+1, r+1)
    long t = (long)(r + 1) * (n0 + 2) + (n0 + 1) - off;
    pad0[r] = (stray && t >= 0 && t < dimp) ? (int)t : -1;
  }
  if (r < n0) {  // dim 1: padded (r+1, n1+1)
    long t = (long)(n1 + 1) * (n0 + 2) + (r + 1) - off;
    pad1[r] = (stray && t >= 0 && t < dimp) ? (int)t : -1;
  }
}

}  // namespace smaug

extern "C" int smaug_euler_step_noalloc(const smaug_params_t* p, const double* w_in, double* w_out,
                                        const double* delx, double* dt, void* stream) {
  using namespace smaug;
  clear_error();
  int rc = validate(p);
  if (rc) return rc;
  if (!w_in || !w_out || !delx || !dt) return set_error(SMAUG_E_INVALID, "null argument");
  if (p->ndim != 2) return set_error(SMAUG_E_UNSUPPORTED, "the allocation-free step is 2D only");
  if (p->precision != SMAUG_PREC_FP64)
    return set_error(SMAUG_E_UNSUPPORTED, "the allocation-free step is FP64 only");
  if (w_in == w_out) return set_error(SMAUG_E_INVALID, "w_in and w_out must not alias");
  if (p->n[0] > NOALLOC_MAXN || p->n[1] > NOALLOC_MAXN)
    return set_error(SMAUG_E_UNSUPPORTED,
                     "grid %d x %d exceeds the allocation-free limit of %d cells per dimension",
                     p->n[0], p->n[1], NOALLOC_MAXN);
  if (p->driver != SMAUG_DRIVER_NONE)
    return set_error(SMAUG_E_UNSUPPORTED, "the allocation-free step has no driver term");
  if (p->boundtype[0][0] == SMAUG_BC_FIXED || p->boundtype[1][0] == SMAUG_BC_FIXED)
    return set_error(SMAUG_E_UNSUPPORTED, "the allocation-free step has no fixed boundaries");
  unsigned char* s = nullptr;
  if ((rc = noalloc_scratch(&s))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long nc = (long)p->n[0] * p->n[1];
  // kernel parameters (same fields as Engine::K)
  KParams K{};
  K.n0 = p->n[0];
  K.n1 = p->n[1];
  K.n2 = 1;
  K.ncell = nc;
  set_boundaries(K, p, 2);
  K.order6 = p->stencil_order == 6;
  for (int d = 0; d < 3; d++) {
    K.dx[d] = p->dx[d];
    K.g[d] = p->g[d];
  }
  K.gamma = p->gamma;
  K.courant = p->courant;
  K.dtmax = p->dtmax;
  for (int f = 0; f < SMAUG_MAXVAR; f++) K.chyp[f] = p->chyp[f];
  K.moddton = p->moddton;
  K.hyperdif = p->hyperdifmom;
  K.has_grav = (p->g[0] != 0.0 || p->g[1] != 0.0);
  K.has_bg = 1;  // exact either way; no host pass over the state
  K.driver = SMAUG_DRIVER_NONE;
  unsigned long long* cm = reinterpret_cast<unsigned long long*>(s + NA_CMAX);
  double* dtb = reinterpret_cast<double*>(s + NA_DT);
  double* tb = reinterpret_cast<double*>(s + NA_T);
  int* flags = reinterpret_cast<int*>(s + NA_FLAGS);
  double* dl = reinterpret_cast<double*>(s + NA_DELX);
  int* pad = reinterpret_cast<int*>(s + NA_PAD);
  // the array keeps the previous call's contents: reset what must start at zero
  CUDA_TRY(cudaMemsetAsync(s, 0, NA_DELX, st));
  CUDA_TRY(cudaMemcpyAsync(dl, delx, sizeof(double) * p->n[0], cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(dl + NOALLOC_MAXN, delx + p->n[0], sizeof(double) * p->n[1],
                           cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(dtb, dt, sizeof(double), cudaMemcpyHostToDevice, st));
  int nmax = p->n[0] > p->n[1] ? p->n[0] : p->n[1];
  noalloc_pad_kernel<<<(nmax + 255) / 256, 256, 0, st>>>(p->n[0], p->n[1],
                                                         p->pad_model == SMAUG_PAD_STRAY, pad,
                                                         pad + NOALLOC_MAXN);
  CUDA_TRY(cudaGetLastError());
  const double* bg = w_in + 6 * nc;
  cmax2d_kernel<<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(K, w_in, bg, cm, 0);
  CUDA_TRY(cudaGetLastError());
  KBufs B{};
  B.uin = w_in;
  B.un = w_in;
  B.uout = w_out;
  B.acc = nullptr;
  B.bg = bg;
  B.delx[0] = dl;
  B.delx[1] = dl + NOALLOC_MAXN;
  B.padsrc[0] = pad;
  B.padsrc[1] = pad + NOALLOC_MAXN;
  B.cmax_in = reinterpret_cast<const double*>(cm);
  B.cmax_out = cm + 3;
  B.cmax_clear = cm + 6;
  B.dt_prev = dtb;
  B.dt_new = dtb + 1;
  B.t_prev = tb;
  B.t_new = tb + 1;
  B.flags = flags;
  B.mode = SMAUG_INT_EULER;
  B.stage = 0;
  CUDA_TRY(stage2d_set_attributes());
  CUDA_TRY(launch_stage2d_any(SMAUG_INT_EULER, false, K, B, st));
  // background fields are constant: carry them to the output
  CUDA_TRY(cudaMemcpyAsync(w_out + 6 * nc, bg, sizeof(double) * 4 * nc, cudaMemcpyDeviceToDevice, st));
  int hflags = 0;
  CUDA_TRY(cudaMemcpyAsync(dt, dtb + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaMemcpyAsync(&hflags, flags, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (hflags & 1) return set_error(SMAUG_E_NONFINITE, "non-finite value in the evolved state");
  return SMAUG_OK;
}
