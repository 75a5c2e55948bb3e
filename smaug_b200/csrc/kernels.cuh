// kernels.cuh -- definitions shared by the engine's translation units:
// tile constants, field numbering, kernel parameter blocks, the precision
// forms and the device helpers of the stage kernels (engine.cu, stage2d.cu,
// stage3d.cu).
#pragma once
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/smaug_b200.h"

namespace smaug {

// ---------------------------------------------------------------------------
// kernel parameters
// ---------------------------------------------------------------------------
// 2D tile shape and the minimum resident blocks per SM of the 2D kernels
// (compile-time; -DSMAUG_TX=.. -DSMAUG_TY=.. -DSMAUG_MINB2D=.. select others)
#ifndef SMAUG_TX
#define SMAUG_TX 32
#endif
#ifndef SMAUG_TY
#define SMAUG_TY 8
#endif
#ifndef SMAUG_MINB2D
#define SMAUG_MINB2D 4
#endif
constexpr int TX = SMAUG_TX;       // tile width (x, fastest)
constexpr int TY = SMAUG_TY;       // tile height
constexpr int HALO = 3;            // stencil radius of the hyperdiffusion windows
constexpr int RX = TX + 2 * HALO;  // staged region
constexpr int RY = TY + 2 * HALO;
constexpr int RC = RX * RY;
constexpr int RXU = RX;            // columns of a region row that the stage reads
constexpr int NTHREADS = TX * TY;
constexpr int XORG = 2;            // x index of the first cell of tile column 0

// 2D field ids (include/iotypes.h:209-216)
enum { RHO = 0, M1 = 1, M2 = 2, EN = 3, B1 = 4, B2 = 5, EB = 6, RHOB = 7, BB1 = 8, BB2 = 9 };

struct KParams {
  int n0, n1, n2;   // n2 = 1 in 2D
  long ncell;
  int bt[3];        // boundtype[dim][0] (upper) -- gradient edge zeroing
  int bc[3];        // ghost-fill type per dim (image pattern; FIXED: no images)
  int gneg[3];      // 1: ghost images along dim are negated (antisymmetric)
  double cmax_floor[3];  // CFL maxima over the fixed ghost cells (constant in time)
  double gamma, courant, dtmax;
  double dx[3];
  double g[3];
  double chyp[SMAUG_MAXVAR];
  int moddton, hyperdif, has_bg, has_grav, driver;
  int order6;       // 1: 6th-order flux derivative (the reference's USE_DORDER3)
  double drv_amp, drv_period, drv_x0[3], drv_sigma[3];
};

// Boundary fields of KParams from the per-dimension types of p.  Ghost images
// follow the reference's generic fills: cont copies the edge cell
// (src/gradops.cu:947-1060), symm/asymm mirror (src/gradops.cu:1325-1465) about
// the face between cells 1 and 2 in 2D and about cell 2 in 3D (the contcd4
// pattern), asymm with the sign flipped; fixed ghost cells are never written
// and keep the values they had when the state was set.
inline void set_boundaries(KParams& K, const smaug_params_t* p, int nd) {
  for (int d = 0; d < 3; d++) {
    const int t = d < nd ? p->boundtype[d][0] : SMAUG_BC_PERIODIC;
    K.bt[d] = t;
    K.bc[d] = (t == SMAUG_BC_SYMM || t == SMAUG_BC_ASYMM) ? (nd == 3 ? SMAUG_BC_CONTCD4 : SMAUG_BC_SYMM) : t;
    K.gneg[d] = (t == SMAUG_BC_ASYMM) ? 1 : 0;
    K.cmax_floor[d] = 0.0;
  }
}

inline bool has_fixed(const KParams& K) {
  return K.bc[0] == SMAUG_BC_FIXED || K.bc[1] == SMAUG_BC_FIXED || K.bc[2] == SMAUG_BC_FIXED;
}

struct KBufs {
  const void* uin;     // [P][ncell] stage input, ghosts valid (double; float in the mixed form)
  const void* un;      // [P][ncell] RK base state (double; its high part in the mixed form)
  const float* un_lo;  // mixed form: low part of the base state
  void* uout;          // [P][ncell] stage output
  float* uout_lo;      // mixed form: low part, written where the output is a base state
  double* acc;         // [P][ncell] RK accumulator (FP64 in both forms)
  const double* bg;    // [B][ncell] background fields (FP64 in both forms)
  const double* delx[3];
  const double* pos[3];
  const int* padsrc[3];
  const double* cmax_in;          // [3]
  unsigned long long* cmax_out;   // [3] (double bits, atomicMax)
  unsigned long long* cmax_clear; // [3] zeroed for the launch after next
  const double* dt_prev;          // dt of the previous step
  double* dt_new;                 // dt of this step (written by stage 0)
  const double* t_prev;
  double* t_new;
  int* flags;
  int mode;   // SMAUG_INT_EULER / SMAUG_INT_RK4
  int stage;  // 0..3
};

// storage and hyperdiffusion arithmetic types of a precision form
template <bool MIX>
struct Form {
  using S = double;  // perturbation storage
  using H = double;  // hyperdiffusion arithmetic
};
template <>
struct Form<true> {
  using S = float;
  using H = float;
};

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
// Loads of a stage's input.  Kernels that run one stage per launch read the
// state through the read-only path (CG = false); a kernel that runs several
// stages in one launch reads what other blocks wrote in an earlier stage of
// the same launch, which only L2 holds coherently, so it loads with .cg
// (CG = true).  ldin: arrays (read-only path by default), ldsc: scalars
// (plain loads by default).
template <bool CG, typename T>
__device__ __forceinline__ T ldin(const T* p) {
  if (CG) return __ldcg(p);
  return __ldg(p);
}
template <bool CG, typename T>
__device__ __forceinline__ T ldsc(const T* p) {
  if (CG) return __ldcg(p);
  return *p;
}
// ---------------------------------------------------------------------------
// bulk tensor copies (TMA) of a staged region into shared memory, completed
// on an mbarrier (the TMA-staged 2D kernel, stage2d_tma.cu)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  // the initialised barrier becomes visible to the copy engine
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// orders the block's earlier shared-memory accesses (made visible to this
// thread by a barrier) before the async copies this thread issues next
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// box of a 3D tensor map ([z][y][x], x fastest) at (x, y, z) into shared
// memory; x * element size must be a multiple of 16 bytes
__device__ __forceinline__ void tma_load_3d(void* dst, const void* map, int x, int y, int z,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
      "%4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
// Wait until the barrier's phase of parity `parity` has completed; false
// when it has not after limit_ns nanoseconds of the global timer.  Each try
// may suspend the thread for up to TRY_WAIT_HINT_NS instead of returning at
// once, so waiting warps do not spin on the shared-memory pipe.
constexpr unsigned TRY_WAIT_HINT_NS = 20000;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, unsigned long long limit_ns) {
  const unsigned a = smem_u32(bar);
  unsigned long long t0 = 0;
  for (unsigned i = 0;; i++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(parity), "r"(TRY_WAIT_HINT_NS)
        : "memory");
    if (done) return true;
    if ((i & 63) == 0) {
      unsigned long long now;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
      if (i == 0)
        t0 = now;
      else if (now - t0 > limit_ns)
        return false;
    }
  }
}
constexpr unsigned long long TMA_WAIT_NS = 2000000000ull;  // 2 s
constexpr int FLAG_TMA_TIMEOUT = 2;                         // KBufs::flags bit

// the bulk-tensor staging of one tile of the TMA-staged 2D kernel
struct TmaTile {
  const void* ms;           // tensor map of the stage input, [field][y][x]
  const void* mg;           // tensor map of the background fields, [field][y][x]
  unsigned long long* bar;  // the block's mbarrier
  unsigned parity;          // phase parity of this tile's copy
  bool issue_self;          // the block's first tile: issue its own copy
  int nbx, nby;             // the block's next tile (nbx < 0: none)
};

__device__ __forceinline__ double dmax0(double m, double v) { return (v > m) ? v : m; }
template <typename T>
__device__ __forceinline__ T hmax0(T m, T v) { return (v > m) ? v : m; }
// quotient of the nu ratio (b > 0): IEEE division in double; in the float
// arithmetic of the mixed form the fast reciprocal-based quotient (2 ulp, far
// below the form's own rounding) for a normal divisor, IEEE division for a
// subnormal one (whose fast reciprocal would overflow)
__device__ __forceinline__ double hdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float hdiv(float a, float b) {
  return b >= 1.17549435e-38f ? __fdividef(a, b) : a / b;
}

// dt rule, src/iosmaug.c:541-616 (a rejected candidate keeps the previous dt,
// see the oracle's dt_rule for why)
__device__ __forceinline__ double device_dt(const KParams& P, const double* cmax, double dt_prev, int nd) {
  if (P.moddton != 1) return dt_prev;
  double courantmax = 1.0e-12;
  double cm = cmax[nd - 1];
  for (int d = 0; d < nd; d++) {
    double t = cm / P.dx[d];
    if (t > courantmax) courantmax = t;
  }
  double dttemp = P.courant / courantmax;
  if (dttemp > 1.0e-12 && dttemp < P.dtmax) return dttemp;
  return dt_prev;
}

// computec3 (src/dervfields.cu:241-309), 2D: the fast speeds along both
// dimensions from one state, sharing 1/rho_t, the pressure and the sound and
// Alfven terms (the reference's divisions by rho_t are multiplications with
// its reciprocal here; the results agree at rounding level)
__device__ __forceinline__ void cfast2_both(double gamma, double rho, double m1, double m2, double e,
                                            double b1, double b2, double eb, double rhob, double bb1,
                                            double bb2, double& c0, double& c1) {
  const double m2s = m1 * m1 + m2 * m2;
  const double b2s = b1 * b1 + b2 * b2;
  const double bbb = bb1 * b1 + bb2 * b2;
  const double bb2s = bb1 * bb1 + bb2 * bb2;
  const double r = 1.0 / (rho + rhob);
  const double pk = (gamma - 1) * (e - 0.5 * (m2s * r) - 0.5 * b2s - bbb);
  const double cs2 = (gamma * (pk + (gamma - 1) * (eb - 0.5 * bb2s))) * r;
  const double cf = (b2s + bb2s + 2.0 * bbb) * r + cs2;
  const double cf2 = cf * cf, k = 4.0 * cs2 * r;
  const double bd0 = bb1 + b1, bd1 = bb2 + b2;
  c0 = sqrt(0.5 * (cf + sqrt(cf2 - k * (bd0 * bd0)))) + fabs(m1 * r);
  c1 = sqrt(0.5 * (cf + sqrt(cf2 - k * (bd1 * bd1)))) + fabs(m2 * r);
}

// the fast speed along `dir` alone
__device__ __forceinline__ double cfast2(double gamma, double rho, double m1, double m2, double e,
                                         double b1, double b2, double eb, double rhob, double bb1,
                                         double bb2, int dir) {
  double c0, c1;
  cfast2_both(gamma, rho, m1, m2, e, b1, b2, eb, rhob, bb1, bb2, c0, c1);
  return dir == 0 ? c0 : c1;
}

// ghost images of interior index a along a dimension of n cells (the
// reference's fill of ghost indices from interior sources, per type)
__device__ __forceinline__ int ghost_images(int a, int n, int type, int* img) {
  int c = 0;
  switch (type) {
    case SMAUG_BC_PERIODIC:
      if (a == n - 4 || a == n - 3) img[c++] = a - (n - 4);
      if (a == 2 || a == 3) img[c++] = a + n - 4;
      break;
    case SMAUG_BC_CONTCD4:
      if (a == 4) img[c++] = 0;
      if (a == 3) img[c++] = 1;
      if (a == n - 4) img[c++] = n - 2;
      if (a == n - 5) img[c++] = n - 1;
      break;
    case SMAUG_BC_CONT:
      if (a == 2) { img[c++] = 0; img[c++] = 1; }
      if (a == n - 3) { img[c++] = n - 2; img[c++] = n - 1; }
      break;
    case SMAUG_BC_SYMM:
      if (a == 3) img[c++] = 0;
      if (a == 2) img[c++] = 1;
      if (a == n - 4) img[c++] = n - 1;
      if (a == n - 3) img[c++] = n - 2;
      break;
    default:
      break;
  }
  return c;
}

// edge zeroing of the gradient operators when boundtype != 0
// (src/gradops.cu:459-474 for grad3dn, :620-823 for the 2nd-order ones;
// evaluated for cells whose other coordinates are inside the band, where the
// reference's precedence-dependent conditions reduce to these sets)
__device__ __forceinline__ bool zero3dn(int a, int n) {
  return a == 2 || a == 3 || a == n - 4 || a == n - 3;
}
__device__ __forceinline__ bool zero1n(int a, int n) {
  return a == 1 || a == 2 || a == n - 3 || a == n - 2;
}

// 3D field ids of the evolved buffer and of the background buffer
enum { R3 = 0, M3 = 1, E3 = 4, B3 = 5 };            // m_c = M3 + c, b_c = B3 + c
enum { GEB = 0, GRB = 1, GBB = 2 };                 // bb_c = GBB + c

// computec3 (src/dervfields.cu:241-309), 3D: the fast speeds along the
// three dimensions, sharing 1/rho_t and the sound and Alfven terms as
// cfast2_both does
__device__ __forceinline__ void cfast3_all(double gamma, const double* s, const double* g, double* c) {
  const double m2s = s[1] * s[1] + s[2] * s[2] + s[3] * s[3];
  const double b2s = s[5] * s[5] + s[6] * s[6] + s[7] * s[7];
  const double bbb = g[2] * s[5] + g[3] * s[6] + g[4] * s[7];
  const double bb2s = g[2] * g[2] + g[3] * g[3] + g[4] * g[4];
  const double r = 1.0 / (s[0] + g[1]);
  const double pk = (gamma - 1) * (s[4] - 0.5 * (m2s * r) - 0.5 * b2s - bbb);
  const double cs2 = (gamma * (pk + (gamma - 1) * (g[0] - 0.5 * bb2s))) * r;
  const double cf = (b2s + bb2s + 2.0 * bbb) * r + cs2;
  const double cf2 = cf * cf, k = 4.0 * cs2 * r;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double bd = g[2 + d] + s[5 + d];
    c[d] = sqrt(0.5 * (cf + sqrt(cf2 - k * (bd * bd)))) + fabs(s[1 + d] * r);
  }
}

// the fast speed along `dir` alone
__device__ __forceinline__ double cfast3(double gamma, const double* s, const double* g, int dir) {
  double c[3];
  cfast3_all(gamma, s, g, c);
  return c[dir];
}

// 4th-order centred derivative along the stride s (grad3dn, src/gradops.cu:437-602)
__device__ __forceinline__ double d4(const double* a, int l, int s, double rdl2) {
  return ((8.0 * (a[l + s] - a[l - s]) + (a[l - 2 * s] - a[l + 2 * s])) * (1.0 / 6.0)) * rdl2;
}

// 6th-order centred derivative of the USE_DORDER3 build (grad3dn,
// src/gradops.cu:450-453): (3 (a+1 - a-1) + 3/5 (a-2 - a+2) - (a-3 - a+3)/15) / 2 / (2 dx)
__device__ __forceinline__ double d6(const double* a, int l, int s, double rdl2) {
  return ((3.0 * (a[l + s] - a[l - s]) + 0.6 * (a[l - 2 * s] - a[l + 2 * s]) -
           (a[l - 3 * s] - a[l + 3 * s]) * (1.0 / 15.0)) * 0.5) * rdl2;
}
// the flux derivative of the selected order
template <bool O6>
__device__ __forceinline__ double dflux(const double* a, int l, int s, double rdl2) {
  return O6 ? d6(a, l, s, rdl2) : d4(a, l, s, rdl2);
}
// cells of the interior where the 6th-order derivative is undefined and
// grad3dn leaves 0: the first and last interior index (x in (2, n-3) only)
__device__ __forceinline__ bool edge6(int a, int n) { return a == 2 || a == n - 3; }

// base state of a field value (the RK4 base / the Euler input) in double
template <bool MIX, bool CG = false>
__device__ __forceinline__ double base_value(const KBufs& B, long idx) {
  if (MIX)
    return (double)ldsc<CG>(static_cast<const float*>(B.un) + idx) + (double)ldsc<CG>(B.un_lo + idx);
  return ldsc<CG>(static_cast<const double*>(B.un) + idx);
}

// store of one stage result; a base state keeps a float high/low pair in the
// mixed form
template <bool MIX>
__device__ __forceinline__ void store_value(const KBufs& B, long idx, double v, bool is_base) {
  if (MIX) {
    const float hi = (float)v;
    static_cast<float*>(B.uout)[idx] = hi;
    if (is_base) B.uout_lo[idx] = (float)(v - (double)hi);
  } else {
    static_cast<double*>(B.uout)[idx] = v;
  }
}

// source interior index of a ghost index (inverse of ghost_images)
__device__ __forceinline__ int ghost_source(int a, int n, int type) {
  if (a >= 2 && a <= n - 3) return a;
  switch (type) {
    case SMAUG_BC_PERIODIC: return (a < 2) ? n - 4 + a : a - n + 4;
    case SMAUG_BC_CONTCD4: return (a < 2) ? 4 - a : (a == n - 1 ? n - 5 : n - 4);
    case SMAUG_BC_CONT: return (a < 2) ? 2 : n - 3;
    case SMAUG_BC_SYMM: return (a < 2) ? 3 - a : 2 * n - 5 - a;
    default: return a;
  }
}


// stage launches (stage2d.cu, stage3d.cu): mode = SMAUG_INT_EULER / _RK4,
// mix = the mixed precision form
cudaError_t launch_stage2d_any(int mode, bool mix, const KParams& K, const KBufs& B, cudaStream_t st);
cudaError_t launch_stage3d_any(int mode, bool mix, const KParams& K, const KBufs& B, cudaStream_t st);
cudaError_t stage2d_set_attributes();
cudaError_t stage3d_set_attributes();
// the fixed ghost layers of a 2D stage, after the stage launch (stage2d.cu)
cudaError_t launch_fixed_ghost2d(int mode, bool mix, const KParams& K, const KBufs& B, cudaStream_t st);

// TMA-staged 2D stage (stage2d_tma.cu).  TmaMap holds an encoded
// CUtensorMap (128 bytes, 64-byte aligned).
struct alignas(64) TmaMap {
  unsigned char bytes[128];
};
// whether the grid admits bulk tensor staging (row pitch a multiple of 16
// bytes in the storage type, no 6th-order stencil)
bool stage2d_tma_supported(const KParams& K, bool mix);
// tensor map of nfield [n1][n0] arrays at base (the stage input: nfield = 6,
// box of all 6; the background fields: box of 4 from field 0 with bg, of
// field 1 alone without); 0 on success
int stage2d_tma_encode(TmaMap* m, const void* base, bool f32, const KParams& K, int nfield, int box_fields);
// persistent: one block per resident slot, each staging its next tile
// during the current one; else one block per tile
cudaError_t launch_stage2d_tma(int mode, bool mix, const KParams& K, const KBufs& B, const TmaMap& ms,
                               const TmaMap& mg, bool persistent, cudaStream_t st);
cudaError_t stage2d_tma_set_attributes();

// Device state of the persistent batch kernel (one launch runs several RK4
// steps of every run): a grid barrier (arrival count, generation) and one
// tile counter per stage; zeroed before every launch.
constexpr int BATCH_MAX_STEPS = 6;
struct BatchSync {
  unsigned int count;
  unsigned int gen;
  int next[4 * BATCH_MAX_STEPS];
};

// batched 2D stages (batch_kernel.cuh), one instantiation per tile shape
// (batch.cu: 32x8, batch16.cu: 16x16): Ks/Bs per run in device memory,
// tiles = (run, tile x, tile y) work list of that shape, `grid` persistent
// blocks
#define SMAUG_BATCH_DECL                                                                        \
  cudaError_t launch_batch2d(int mode, bool mix, const KParams* Ks, const KBufs* Bs,           \
                             const int4* tiles, int ntiles, int grid, cudaStream_t st);         \
  cudaError_t launch_batch2d_cycle(bool mix, const KParams* Ks, const KBufs* Bs,              \
                                   const int4* tiles, int ntiles, int nruns, int k0,           \
                                   int nsteps, BatchSync* sync, int* err, int grid,            \
                                   cudaStream_t st);                                            \
  cudaError_t batch2d_set_attributes();                                                         \
  int batch2d_max_blocks_per_sm(bool mix);                                                      \
  int batch2d_cycle_max_blocks_per_sm(bool mix);
namespace t32x8 { SMAUG_BATCH_DECL }
namespace t16x16 { SMAUG_BATCH_DECL }
#undef SMAUG_BATCH_DECL

}  // namespace smaug
