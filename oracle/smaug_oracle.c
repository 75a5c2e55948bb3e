/*
 * smaug_oracle.c -- CPU FP64 restatement of SMAUG's single-GPU time advance.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * engine in smaug_b200/csrc; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.  The product never calls it.
 *
 * It restates, kernel by kernel and in the reference's launch order, the
 * arithmetic of mikeg64/smaug (paths relative to the project root):
 *   driver step sequence     src/iosmaug.c:496-835 (rkon==0 branch)
 *   derived fields           src/dervfields.cu:46-309
 *   gradient operators       src/gradops.cu:437-823
 *   mass/momentum fluxes     src/centdiff1.cu:19-580
 *   energy/induction fluxes  src/centdiff2.cu:19-1171
 *   CFL max                  src/computedervfields.cu:1457-1533,1864-2050
 *   hyperdiffusion nu        src/hyperdifvisc1r.cu:426-1413, src/hyperdifvisc1l.cu:17-1423
 *   hyperdiffusive sources   src/hyperdif{rho,e,mom,momne,b,bne}source1.cu
 *   ghost cells              src/boundary.cu:72-252, src/gradops.cu:833-1465
 *   grid metric              src/init.cu:2502-3060
 * Every loop below is one reference __global__ kernel: the reference runs one
 * thread per cell with a host synchronisation after each launch, so a
 * sequential loop over cells reproduces it wherever threads of one launch do
 * not race.  The one racing launch (the stray wtemp2 store in
 * hyperdifvisc1r_parallel, src/hyperdifvisc1r.cu:1235,1255) is modelled
 * explicitly by params->pad_model.
 *
 * Parity status: pinned against the reference binary built from the
 * reference's own sources (oracle/build_ref.py) and run on a B200; see the
 * golden fixtures under tests/golden/.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/smaug_b200.h"

#ifdef _OPENMP
#include <omp.h>
#define PFOR _Pragma("omp parallel for schedule(static)")
#else
#define PFOR
#endif

#define SMALLDOUBLE 1.0e-12 /* include/iotypes.h:21 */

/* -------------------------------------------------------------------------
 * Workspace and index helpers (src/gradops.cu:44-97)
 * ---------------------------------------------------------------------- */
typedef struct {
  const smaug_params_t *P;
  int nd;         /* NDIM */
  int n[3];       /* n[2]==1 in 2D */
  long dimp;
  int nvar, nderv;
  /* field ids (include/iotypes.h:209-230) */
  int rho, mom[3], energy, b[3], energyb, rhob, bb[3];
  int vel[3], flux, hdnur, hdnul, nushk[3], soundspeed, pressuret, pressurek,
      bdotv, cfast, ptb, pkb, pos[3], delx[3];
  long p1n[3], p1size, p2n[3], p2size;
  double *w0, *w1;       /* slots order=0 and ordero=1 (NVAR*dimp each) */
  double *wd;            /* NDERV*dimp */
  double *wtemp;         /* NTEMP=8 * dimp */
  double *wtemp1;        /* NTEMP1=2 * p1size */
  double *wtemp2;        /* NTEMP2=1 * p2size */
  double *dwn1;          /* NVAR*dimp */
  double dt;             /* p->dt */
  double cmax;           /* p->cmax */
  double t;              /* simulated time, for the driver phase */
  long it;               /* step counter (the reference's p->it = n) */
  int increment_mode;    /* slot1 starts at 0 for evolved fields (RK4 stages) */
} O;

enum { tmp1 = 0, tmp2, tmp3, tmp4, tmp5, tmp6, tmp7, tmp8 };
enum { d1 = 0, d3 = 1 };

static inline long E(const O *o, int i, int j, int k) {
  return ((long)k * o->n[1] + j) * o->n[0] + i;
}
static inline long F(const O *o, int f) { return (long)f * o->dimp; }
/* encode3p1 / encode3p2: in 2D the k argument is ignored (src/gradops.cu:56-85) */
static inline long E1(const O *o, int i, int j, int k, int f) {
  if (o->nd == 2) k = 0;
  return ((long)k * o->p1n[1] + j) * o->p1n[0] + i + (long)f * o->p1size;
}
static inline long E2(const O *o, int i, int j, int k, int f) {
  if (o->nd == 2) k = 0;
  return ((long)k * o->p2n[1] + j) * o->p2n[0] + i + (long)f * o->p2size;
}
static inline int kofs(const O *o, int a) { return o->nd == 3 ? a : 0; }

#define FOR_CELLS(o)                                                  \
  PFOR for (long _c = 0; _c < (o)->dimp; _c++) {                      \
    int ii[3];                                                        \
    ii[0] = (int)(_c % (o)->n[0]);                                    \
    ii[1] = (int)((_c / (o)->n[0]) % (o)->n[1]);                      \
    ii[2] = (int)(_c / ((long)(o)->n[0] * (o)->n[1]));                \
    const int i = ii[0], j = ii[1], k = ii[2];                        \
    (void)i; (void)j; (void)k;
#define END_CELLS }

static void setup_ids(O *o) {
  int nd = o->nd;
  o->nvar = 4 + 3 * nd;
  o->nderv = 4 * nd + 11;
  o->rho = 0;
  for (int d = 0; d < 3; d++) {
    o->mom[d] = 1 + d;
    o->b[d] = 2 + nd + d;
    o->bb[d] = 4 + 2 * nd + d;
    o->vel[d] = d;
    o->nushk[d] = nd + 3 + d;
    o->pos[d] = 2 * nd + 11 + d;
    o->delx[d] = 3 * nd + 11 + d;
  }
  o->energy = 1 + nd;
  o->energyb = 2 + 2 * nd;
  o->rhob = 3 + 2 * nd;
  o->flux = nd;
  o->hdnur = nd + 1;
  o->hdnul = nd + 2;
  o->soundspeed = 2 * nd + 3;
  o->pressuret = 2 * nd + 4;
  o->pressurek = 2 * nd + 5;
  o->bdotv = 2 * nd + 6;
  o->cfast = 2 * nd + 8;
  o->ptb = 2 * nd + 9;
  o->pkb = 2 * nd + 10;
}

static int init_O(O *o, const smaug_params_t *P) {
  memset(o, 0, sizeof(*o));
  o->P = P;
  o->nd = P->ndim;
  if (o->nd != 2 && o->nd != 3) return SMAUG_E_INVALID;
  o->n[0] = P->n[0];
  o->n[1] = P->n[1];
  o->n[2] = (o->nd == 3) ? P->n[2] : 1;
  for (int d = 0; d < o->nd; d++)
    if (o->n[d] < 8) return SMAUG_E_INVALID;
  o->dimp = (long)o->n[0] * o->n[1] * o->n[2];
  setup_ids(o);
  for (int d = 0; d < 3; d++) {
    o->p1n[d] = (d < o->nd) ? o->n[d] + 1 : 1;
    o->p2n[d] = (d < o->nd) ? o->n[d] + 2 : 1;
  }
  o->p1size = o->p1n[0] * o->p1n[1] * o->p1n[2];
  o->p2size = o->p2n[0] * o->p2n[1] * o->p2n[2];
  o->w0 = calloc((size_t)o->nvar * o->dimp, sizeof(double));
  o->w1 = calloc((size_t)o->nvar * o->dimp, sizeof(double));
  o->wd = calloc((size_t)o->nderv * o->dimp, sizeof(double));
  o->wtemp = calloc((size_t)8 * o->dimp, sizeof(double));
  o->wtemp1 = calloc((size_t)2 * o->p1size, sizeof(double));
  o->wtemp2 = calloc((size_t)o->p2size, sizeof(double));
  o->dwn1 = calloc((size_t)o->nvar * o->dimp, sizeof(double));
  if (!o->w0 || !o->w1 || !o->wd || !o->wtemp || !o->wtemp1 || !o->wtemp2 ||
      !o->dwn1)
    return SMAUG_E_NOMEM;
  return 0;
}

static void free_O(O *o) {
  free(o->w0); free(o->w1); free(o->wd); free(o->wtemp);
  free(o->wtemp1); free(o->wtemp2); free(o->dwn1);
}

static inline int bt0(const O *o, int dir) { return o->P->boundtype[dir][0]; }

/* ---- gradient operators (src/gradops.cu:437-823) ---------------------- */

/* all coordinates except `dir` satisfy lo < c < n-hi */
static inline int others_in(const O *o, const int *ii, int dir, int lo, int hi) {
  for (int d = 0; d < o->nd; d++) {
    if (d == dir) continue;
    if (!(ii[d] > lo && ii[d] < o->n[d] - hi)) return 0;
  }
  return 1;
}

static inline long stepd(const O *o, int dir) {
  return dir == 0 ? 1 : (dir == 1 ? o->n[0] : (long)o->n[0] * o->n[1]);
}

/* grad3dn_MODID: 4th-order centred derivative, src/gradops.cu:437-602; the
   6th-order form of the USE_DORDER3 build (stencil_order 6,
   src/gradops.cu:450-453) is defined on x in (2, n-3) only.  In 2D the
   reference's dir-1 branch has no #else after its USE_DORDER3 block
   (src/gradops.cu:536-544): the 4th-order form that follows overwrites it,
   so a 2D build is 6th order along dim 0 and 4th order along dim 1. */
static double grad3dn(const O *o, const double *a, const int *ii, int field, int dir) {
  double grad = 0;
  int x = ii[dir], n = o->n[dir];
  long c = E(o, ii[0], ii[1], ii[2]);
  long s = stepd(o, dir);
  if (o->P->stencil_order == 6 && !(o->nd == 2 && dir == 1)) {
    if (x > 2 && x < n - 3)
      grad = (((3 * a[c + s] - 3 * a[c - s] + 3.0 * (a[c - 2 * s] - a[c + 2 * s]) / 5.0 -
                (a[c - 3 * s] - a[c + 3 * s]) / 15.0) / 2.0)) /
             (2.0 * (o->wd[F(o, o->delx[dir]) + c]));
  } else if (x > 1 && x < n - 2) {
    grad = ((8 * a[c + s] - 8 * a[c - s] + a[c - 2 * s] - a[c + 2 * s]) / 6.0) /
           (2.0 * (o->wd[F(o, o->delx[dir]) + c]));
  }
  (void)field;
  if (bt0(o, dir) != 0) {
    /* C precedence: a || (b && c && ...) (src/gradops.cu:463-474) */
    int oth = others_in(o, ii, dir, 1, 2);
    if ((x == n - 3) || ((x == n - 4) && oth))
      grad = 0;
    else if (x == 2 || ((x == 3) && oth))
      grad = 0;
  }
  return grad;
}

/* edge-zeroing of the one-sided operators; the reference's conditions for
   the other coordinates are j>0 && j<n-1 (and a k>1 typo in grad1l3n dir 0
   3D, src/gradops.cu:626) */
static int onesided_zero(const O *o, const int *ii, int dir, int first_klo) {
  int x = ii[dir], n = o->n[dir];
  int oth1 = 1, oth2 = 1;
  for (int d = 0; d < o->nd; d++) {
    if (d == dir) continue;
    int lo1 = 0;
    if (o->nd == 3 && d == 2 && dir == 0) lo1 = first_klo;
    if (!(ii[d] > lo1 && ii[d] < o->n[d] - 1)) oth1 = 0;
    if (!(ii[d] > 0 && ii[d] < o->n[d] - 1)) oth2 = 0;
  }
  if ((x == n - 2) || ((x == n - 3) && oth1)) return 1;
  if (x == 1 || ((x == 2) && oth2)) return 1;
  return 0;
}

/* grad1l3n_MODID, src/gradops.cu:608-677 */
static double grad1l3n(const O *o, const double *a, const int *ii, int dir) {
  double grad = 0;
  int x = ii[dir];
  long c = E(o, ii[0], ii[1], ii[2]);
  long s = stepd(o, dir);
  if (x > 0 && x < o->n[dir]) {
    grad = (a[c] - a[c - s]) / (o->wd[F(o, o->delx[dir]) + c]);
    if (bt0(o, dir) != 0 && onesided_zero(o, ii, dir, 1)) grad = 0;
  }
  return grad;
}

/* grad1r3n_MODID, src/gradops.cu:680-750 */
static double grad1r3n(const O *o, const double *a, const int *ii, int dir) {
  double grad = 0;
  int x = ii[dir];
  long c = E(o, ii[0], ii[1], ii[2]);
  long s = stepd(o, dir);
  if (x < o->n[dir] - 1) {
    grad = (a[c + s] - a[c]) / (o->wd[F(o, o->delx[dir]) + c]);
    if (bt0(o, dir) != 0 && onesided_zero(o, ii, dir, 0)) grad = 0;
  }
  return grad;
}

/* grad13n_MODID, src/gradops.cu:755-823 */
static double grad13n(const O *o, const double *a, const int *ii, int dir) {
  double grad = 0;
  int x = ii[dir];
  long c = E(o, ii[0], ii[1], ii[2]);
  long s = stepd(o, dir);
  if (x > 0 && x < o->n[dir] - 1) {
    grad = ((a[c + s] - a[c - s]) / (o->wd[F(o, o->delx[dir]) + c])) / 2.0;
    if (bt0(o, dir) != 0 && onesided_zero(o, ii, dir, 0)) grad = 0;
  }
  return grad;
}

/* ---- derived fields (src/dervfields.cu) ------------------------------- */
#define W(f) (w[F(o, (f)) + c])

/* computevel3_MODID, src/dervfields.cu:79-98 */
static void computevel3(O *o, const double *w, long c) {
  for (int d = 0; d < o->nd; d++)
    o->wd[F(o, o->vel[d]) + c] = W(o->mom[d]) / (W(o->rho) + W(o->rhob));
}

/* computept3_MODID, src/dervfields.cu:107-153 */
static void computept3(O *o, const double *w, long c) {
  double g = o->P->gamma;
  double bb = 0, b2 = 0, m2 = 0;
  for (int d = 0; d < o->nd; d++) {
    bb = (d == 0) ? W(o->b[0]) * W(o->bb[0]) : bb + W(o->b[d]) * W(o->bb[d]);
    b2 = (d == 0) ? W(o->b[0]) * W(o->b[0]) : b2 + W(o->b[d]) * W(o->b[d]);
    m2 = (d == 0) ? W(o->mom[0]) * W(o->mom[0]) : m2 + W(o->mom[d]) * W(o->mom[d]);
  }
  double pt = (g - 2.0) * (bb + 0.5 * b2);
  pt = (g - 1.0) * (W(o->energy) - 0.5 * m2 / (W(o->rho) + W(o->rhob))) - pt;
  o->wd[F(o, o->pressuret) + c] = pt;
}

/* computepbg3_MODID, src/dervfields.cu:157-191 */
static double pbg_value(const O *o, const double *w, long c) {
  double g = o->P->gamma;
  double s = 0;
  for (int d = 0; d < o->nd; d++)
    s = (d == 0) ? W(o->bb[0]) * W(o->bb[0]) : s + W(o->bb[d]) * W(o->bb[d]);
  return (g - 1) * W(o->energyb) - 0.5 * (g - 2) * s;
}

/* computec3_MODID, src/dervfields.cu:241-309 */
static void computec3(O *o, const double *w, long c, int dir) {
  double g = o->P->gamma;
  double m2 = 0, b2 = 0, bbb = 0, bb2 = 0;
  for (int d = 0; d < o->nd; d++) {
    m2 = (d == 0) ? W(o->mom[0]) * W(o->mom[0]) : m2 + W(o->mom[d]) * W(o->mom[d]);
    b2 = (d == 0) ? W(o->b[0]) * W(o->b[0]) : b2 + W(o->b[d]) * W(o->b[d]);
    bbb = (d == 0) ? W(o->bb[0]) * W(o->b[0]) : bbb + W(o->bb[d]) * W(o->b[d]);
    bb2 = (d == 0) ? W(o->bb[0]) * W(o->bb[0]) : bb2 + W(o->bb[d]) * W(o->bb[d]);
  }
  double rt = W(o->rho) + W(o->rhob);
  double pk = (g - 1) * (W(o->energy) - 0.5 * (m2 / rt) - 0.5 * b2 - bbb);
  double cs2 = (g * (pk + (g - 1) * (W(o->energyb) - 0.5 * bb2))) / rt;
  double cf = (b2 + bb2 + 2.0 * bbb) / rt + cs2;
  double bd = W(o->bb[dir]) + W(o->b[dir]);
  double cfasti = 0.5 * (cf + sqrt(cf * cf - 4.0 * cs2 * (bd * bd) / rt));
  o->wd[F(o, o->cfast) + c] = sqrt(cfasti) + fabs(W(o->mom[dir]) / rt);
  o->wd[F(o, o->soundspeed) + c] = sqrt(cs2);
}
#undef W

/* strip of the directional derived-field/flux kernels: every coordinate but
   dir in [2, n-3] (src/computedervfields.cu:80-107) */
static inline int in_strip(const O *o, const int *ii, int dir) {
  return others_in(o, ii, dir, 1, 2);
}
static inline int in_interior(const O *o, const int *ii) {
  for (int d = 0; d < o->nd; d++)
    if (!(ii[d] > 1 && ii[d] < o->n[d] - 2)) return 0;
  return 1;
}
static inline int in_band1(const O *o, const int *ii) {
  for (int d = 0; d < o->nd; d++)
    if (!(ii[d] > 0 && ii[d] < o->n[d] - 1)) return 0;
  return 1;
}

/* cucomputevels (src/computedervfields.cu:18-126) */
static void k_computevels(O *o, int dir) {
  FOR_CELLS(o)
  if (in_strip(o, ii, dir)) computevel3(o, o->w0, _c);
  END_CELLS
}

/* cucomputept: computeptzero_parallel + computept_parallel
   (src/computedervfields.cu:129-388, wrapper :2266-2298) */
static void k_computept(O *o, int dir) {
  FOR_CELLS(o)
  o->wd[F(o, o->pressuret) + _c] = 0.0;
  END_CELLS
  FOR_CELLS(o)
  if (in_strip(o, ii, dir)) computept3(o, o->w0, _c);
  END_CELLS
}

/* cucomputepbg (src/computedervfields.cu:527-661) */
static void k_computepbg(O *o, const double *w) {
  FOR_CELLS(o)
  o->wd[F(o, o->ptb) + _c] = pbg_value(o, w, _c);
  END_CELLS
}

/* cucomputec + cucomputemaxc: global max of cfast over all cells, ghosts
   included (src/computedervfields.cu:1457-1533,1864-2050); the sound-speed
   pass of cucomputemaxc reduces a zeroed buffer and contributes 0. */
static double k_cmax(O *o, int dir) {
  double m = 0.0;
  FOR_CELLS(o)
  computec3(o, o->w0, _c, dir);
  END_CELLS
  for (long c = 0; c < o->dimp; c++) {
    double v = o->wd[F(o, o->cfast) + c];
    if (v > m) m = v;
  }
  return m;
}

/* ---- centdiff1 (src/centdiff1.cu) -------------------------------------- */
static double transportflux(const O *o, const double *w, long c, int field, int d) {
  return w[F(o, o->mom[d]) + c] * w[F(o, field) + c] /
         (w[F(o, o->rho) + c] + w[F(o, o->rhob) + c]);
}

static void computeflux_cd1(O *o, const double *w, long c, int field, int d) {
  double *fx = &o->wd[F(o, o->flux) + c];
  if (field == o->rho) {
    /* computefluxrho, src/centdiff1.cu:133-147 */
    *fx = transportflux(o, w, c, o->rho, d) +
          (w[F(o, o->rhob) + c] * w[F(o, o->mom[d]) + c]) /
              (w[F(o, o->rhob) + c] + w[F(o, o->rho) + c]);
  } else {
    /* computefluxmom1/2/3 + fluxmom1{0,1,2}, src/centdiff1.cu:82-197 */
    int cmp = field - o->mom[0];
    double bf = w[F(o, o->b[cmp]) + c], bbf = w[F(o, o->bb[cmp]) + c];
    double bbd = w[F(o, o->bb[d]) + c], bd = w[F(o, o->b[d]) + c];
    double fm;
    if (d == cmp)
      fm = o->wd[F(o, o->pressuret) + c] - (bf * bbd + bbf * bd) - bf * bd;
    else
      fm = -(bf * bbd + bbf * bd) - bf * bd;
    *fx = 0.0;
    *fx += transportflux(o, w, c, field, d) + fm;
  }
}

/* cucentdiff1, src/centdiff1.cu:822-851 */
static void k_centdiff1(O *o, int f, int dir) {
  FOR_CELLS(o)
  o->dwn1[F(o, f) + _c] = 0.0;
  o->wd[F(o, o->flux) + _c] = 0.0;
  END_CELLS
  FOR_CELLS(o)
  if (in_strip(o, ii, dir)) computeflux_cd1(o, o->w0, _c, f, dir);
  END_CELLS
  FOR_CELLS(o)
  if (in_interior(o, ii))
    o->dwn1[F(o, f) + _c] += grad3dn(o, &o->wd[F(o, o->flux)], ii, o->flux, dir);
  END_CELLS
  FOR_CELLS(o)
  if (in_strip(o, ii, dir))
    o->w1[F(o, f) + _c] = o->w1[F(o, f) + _c] - o->dt * o->dwn1[F(o, f) + _c];
  END_CELLS
}

/* ---- centdiff2 (src/centdiff2.cu) -------------------------------------- */
static double fluxe1(const O *o, const double *w, long c, int d) {
  /* src/centdiff2.cu:203-243 */
  double bbm = 0, bm = 0;
  for (int a = 0; a < o->nd; a++) {
    bbm = (a == 0) ? w[F(o, o->bb[0]) + c] * w[F(o, o->mom[0]) + c]
                   : bbm + w[F(o, o->bb[a]) + c] * w[F(o, o->mom[a]) + c];
    bm = (a == 0) ? w[F(o, o->b[0]) + c] * w[F(o, o->mom[0]) + c]
                  : bm + w[F(o, o->b[a]) + c] * w[F(o, o->mom[a]) + c];
  }
  double rt = w[F(o, o->rho) + c] + w[F(o, o->rhob) + c];
  double md = w[F(o, o->mom[d]) + c];
  double ft = md * (o->wd[F(o, o->pressuret) + c]);
  ft -= w[F(o, o->b[d]) + c] * bbm;
  ft -= w[F(o, o->bb[d]) + c] * bm;
  ft /= rt;
  ft += md * w[F(o, o->energyb) + c] / rt;
  ft -= w[F(o, o->b[d]) + c] * bm / rt;
  return ft;
}

static void computeflux_cd2(O *o, const double *w, long c, int field, int d) {
  double *fx = &o->wd[F(o, o->flux) + c];
  *fx = 0.0;
  if (field == o->energy) {
    /* computefluxe, src/centdiff2.cu:253-264 */
    *fx = transportflux(o, w, c, o->energy, d) + fluxe1(o, w, c, d);
  } else {
    /* computefluxb1/b2/b3, src/centdiff2.cu:267-323 */
    int cmp = field - o->b[0];
    if (d == cmp) {
      *fx = 0.0;
    } else {
      double rt = w[F(o, o->rho) + c] + w[F(o, o->rhob) + c];
      *fx = transportflux(o, w, c, field, d) -
            (w[F(o, o->b[d]) + c] + w[F(o, o->bb[d]) + c]) * w[F(o, o->mom[cmp]) + c] / rt +
            (w[F(o, o->bb[cmp]) + c]) * w[F(o, o->mom[d]) + c] / rt;
    }
  }
}

/* cucentdiff2, src/centdiff2.cu:1117-1171 */
static void k_centdiff2(O *o, int f, int dir) {
  FOR_CELLS(o)
  o->dwn1[F(o, f) + _c] = 0.0;
  o->wd[F(o, o->flux) + _c] = 0.0;
  END_CELLS
  FOR_CELLS(o)
  if (in_strip(o, ii, dir)) computeflux_cd2(o, o->w0, _c, f, dir);
  END_CELLS
  FOR_CELLS(o) /* centdiff2a */
  if (in_interior(o, ii))
    o->dwn1[F(o, f) + _c] = grad3dn(o, &o->wd[F(o, o->flux)], ii, o->flux, dir);
  END_CELLS
  FOR_CELLS(o) /* centdiff2b */
  if (in_strip(o, ii, dir))
    o->w1[F(o, f) + _c] = o->w1[F(o, f) + _c] - o->dt * o->dwn1[F(o, f) + _c];
  END_CELLS
  /* centdiff2ci: background total pressure from slot ordero, dwn1 reset */
  k_computepbg(o, o->w1);
  FOR_CELLS(o)
  o->dwn1[F(o, f) + _c] = 0.0;
  END_CELLS
  /* centdiff2c: addenergyterms_cd2 (src/centdiff2.cu:80-115,587-717); the 2D
     launch bound has no lower limit (i<n0-2 && j<n1-2) */
  if (f != o->energy) return;
  FOR_CELLS(o)
  int ok;
  if (o->nd == 2)
    ok = (i < o->n[0] - 2 && j < o->n[1] - 2);
  else
    ok = in_interior(o, ii);
  if (ok) {
    double *e = &o->w1[F(o, o->energy) + _c];
    *e -= +(o->dt) * o->wd[F(o, o->ptb) + _c] *
          grad3dn(o, &o->wd[F(o, o->vel[dir])], ii, o->vel[dir], dir);
    for (int idim = 0; idim < o->nd; idim++)
      *e += (o->dt) * o->w1[F(o, o->bb[idim]) + _c] * o->w1[F(o, o->bb[dir]) + _c] *
            grad3dn(o, &o->wd[F(o, o->vel[dir])], ii, o->vel[dir], idim);
  }
  END_CELLS
}

/* cugrav: addgrav_cd2 (src/centdiff2.cu:118-154,721-787, wrapper :1174-1209) */
static void k_grav(O *o) {
  FOR_CELLS(o)
  int ok;
  if (o->nd == 2)
    ok = (i < o->n[0] - 2 && j < o->n[1] - 2);
  else
    ok = in_interior(o, ii);
  if (ok) {
    const double *w = o->w0;
    for (int d = 0; d < o->nd; d++)
      o->w1[F(o, o->mom[d]) + _c] += (o->dt) * (o->P->g[d]) * w[F(o, o->rho) + _c];
    for (int d = 0; d < o->nd; d++)
      o->w1[F(o, o->energy) + _c] +=
          (o->dt) * w[F(o, o->rho) + _c] * ((o->P->g[d]) * w[F(o, o->mom[d]) + _c]) /
          (w[F(o, o->rho) + _c] + w[F(o, o->rhob) + _c]);
  }
  END_CELLS
}

/* ---- hyperdiffusion coefficient (src/hyperdifvisc1r.cu, 1l.cu) -------- */

/* q of the (field) for hyperviscosity: hyperdifvisc1r_parallel tmp6
   (src/hyperdifvisc1r.cu:1225-1253) */
static double hq(const O *o, const double *w, long c, int field) {
  if (field == o->energy) {
    double b2 = 0, m2 = 0;
    for (int d = 0; d < o->nd; d++) {
      b2 = (d == 0) ? w[F(o, o->b[0]) + c] * w[F(o, o->b[0]) + c]
                    : b2 + w[F(o, o->b[d]) + c] * w[F(o, o->b[d]) + c];
      m2 = (d == 0) ? w[F(o, o->mom[0]) + c] * w[F(o, o->mom[0]) + c]
                    : m2 + w[F(o, o->mom[d]) + c] * w[F(o, o->mom[d]) + c];
    }
    return w[F(o, o->energy) + c] -
           0.5 * (b2 + m2 / (w[F(o, o->rho) + c] + w[F(o, o->rhob) + c]));
  }
  double v = w[F(o, field) + c];
  if (field >= o->mom[0] && field <= o->mom[o->nd - 1])
    v = w[F(o, field) + c] / ((w[F(o, o->rho) + c] + w[F(o, o->rhob) + c]));
  return v;
}

/* zeroing part of hyperdifvisc1{r,l}_parallel (src/hyperdifvisc1r.cu:1099-1188) */
static void visc_zero(O *o) {
  FOR_CELLS(o)
  for (int f = tmp1; f <= tmp8; f++) o->wtemp[F(o, f) + _c] = 0;
  for (int f = d1; f <= d3; f++) o->wtemp1[E1(o, i, j, k, f)] = 0;
  o->wtemp2[E2(o, i, j, k, 0)] = 0;
  END_CELLS
  /* padded edges (the i==n0-1 / j==n1-1 / k==n2-1 branches) */
  long p2 = o->p2size;
  (void)p2;
  for (long c = 0; c < o->dimp; c++) {
    int i = (int)(c % o->n[0]);
    int j = (int)((c / o->n[0]) % o->n[1]);
    int k = (int)(c / ((long)o->n[0] * o->n[1]));
    int ni = o->n[0], nj = o->n[1], nk = o->n[2];
    if (i == ni - 1) {
      for (int f = d1; f <= d3; f++) o->wtemp1[E1(o, i + 1, j, k, f)] = 0;
      o->wtemp2[E2(o, i + 1, j, k, 0)] = 0;
      o->wtemp2[E2(o, i + 2, j, k, 0)] = 0;
    }
    if (j == nj - 1) {
      for (int f = d1; f <= d3; f++) o->wtemp1[E1(o, i, j + 1, k, f)] = 0;
      o->wtemp2[E2(o, i, j + 1, k, 0)] = 0;
      o->wtemp2[E2(o, i, j + 2, k, 0)] = 0;
    }
    if (o->nd == 3 && k == nk - 1) {
      for (int f = d1; f <= d3; f++) o->wtemp1[E1(o, i, j, k + 1, f)] = 0;
      o->wtemp2[E2(o, i, j, k + 1, 0)] = 0;
      o->wtemp2[E2(o, i, j, k + 2, 0)] = 0;
    }
    if (j == nj - 1 && i == ni - 1) {
      for (int f = d1; f <= d3; f++) o->wtemp1[E1(o, i + 1, j + 1, k, f)] = 0;
      for (int di = 0; di < 2; di++)
        for (int dj = 0; dj < 2; dj++) o->wtemp2[E2(o, i + 1 + di, j + 1 + dj, k, 0)] = 0;
    }
    if (o->nd == 3 && i == ni - 1 && k == nk - 1) {
      for (int f = d1; f <= d3; f++) o->wtemp1[E1(o, i + 1, j, k + 1, f)] = 0;
      for (int di = 0; di < 2; di++)
        for (int dk = 0; dk < 2; dk++) o->wtemp2[E2(o, i + 1 + di, j, k + 1 + dk, 0)] = 0;
    }
    if (o->nd == 3 && j == nj - 1 && k == nk - 1) {
      for (int f = d1; f <= d3; f++) o->wtemp1[E1(o, i + 1, j + 1, k, f)] = 0;
      for (int dk = 0; dk < 2; dk++)
        for (int dj = 0; dj < 2; dj++) o->wtemp2[E2(o, i, j + 1 + dj, k + 1 + dk, 0)] = 0;
    }
    if (o->nd == 3 && i == ni - 1 && j == nj - 1 && k == nk - 1) {
      for (int f = d1; f <= d3; f++) o->wtemp1[E1(o, i + 1, j + 1, k + 1, f)] = 0;
      for (int dk = 0; dk < 2; dk++)
        for (int dj = 0; dj < 2; dj++)
          for (int di = 0; di < 2; di++)
            o->wtemp2[E2(o, i + 1 + di, j + 1 + dj, k + 1 + dk, 0)] = 0;
    }
  }
}

/* The right-biased first kernel also stores tmp6 through encode3 instead of
   encode3p2 (src/hyperdifvisc1r.cu:1235,1255): linear index (k+1)n0n1 +
   (j+1)n0 + (i+1) of the padded array.  Those stores race with the zeroing
   of the same launch; pad_model selects which store is taken to land last.
   Interior padded positions are rewritten by hyperdifvisc1ar afterwards, so
   only pad positions keep the stray values. */
static void visc_stray_store(O *o) {
  if (o->P->pad_model != SMAUG_PAD_STRAY) return;
  for (long c = 0; c < o->dimp; c++) {
    int i = (int)(c % o->n[0]);
    int j = (int)((c / o->n[0]) % o->n[1]);
    int k = (int)(c / ((long)o->n[0] * o->n[1]));
    long lin;
    if (o->nd == 3)
      lin = (long)(k + 1) * o->n[0] * o->n[1] + (long)(j + 1) * o->n[0] + (i + 1);
    else
      lin = (long)(j + 1) * o->n[0] + (i + 1);
    if (lin < o->p2size) o->wtemp2[lin] = o->wtemp[F(o, tmp6) + c];
  }
}

/* hyperdifvisc1r_parallel / hyperdifvisc1l_parallel */
static void k_visc1(O *o, int field, int right) {
  visc_zero(o);
  FOR_CELLS(o)
  o->wtemp[F(o, tmp6) + _c] = hq(o, o->w0, _c, field);
  END_CELLS
  if (right) visc_stray_store(o);
  FOR_CELLS(o)
  o->wd[F(o, right ? o->hdnur : o->hdnul) + _c] = 0;
  END_CELLS
}

/* hyperdifvisc1ar/1al: copy tmp6 into the padded array */
static void k_visc1a(O *o) {
  FOR_CELLS(o)
  o->wtemp2[E2(o, i + 1, j + 1, k + kofs(o, 1), 0)] = o->wtemp[F(o, tmp6) + _c];
  END_CELLS
}

/* hyperdifvisc1bcl: bc_hyperdifl pad fill (src/hyperdifvisc1l.cu:17-62) */
static void k_visc1bcl(O *o, int dim) {
  int is = 1;
  FOR_CELLS(o)
  int ni = o->n[0], nj = o->n[1], nk = o->n[2];
  if (o->nd == 2) {
    if ((dim == 0) && (i == ni - 1))
      o->wtemp2[E2(o, i + 2, j + is, 0, 0)] = o->wtemp2[E2(o, ni - 5, j + is, 0, 0)];
    else if ((dim == 1) && (j == nj - 1))
      o->wtemp2[E2(o, i + is, j + 2, 0, 0)] = o->wtemp2[E2(o, i + is, nj - 5, 0, 0)];
    else if ((dim == 0) && (i == 0))
      o->wtemp2[E2(o, 0, j + is, 0, 0)] = o->wtemp2[E2(o, 6, j + is, 0, 0)];
    else if ((dim == 1) && (j == 0))
      o->wtemp2[E2(o, i + is, 0, 0, 0)] = o->wtemp2[E2(o, i + is, 6, 0, 0)];
  } else {
    if ((dim == 0) && (i == ni - 1))
      o->wtemp2[E2(o, i + 2, j + is, k + is, 0)] = o->wtemp2[E2(o, ni - 5, j + is, k + is, 0)];
    else if ((dim == 1) && (j == nj - 1))
      o->wtemp2[E2(o, i + is, j + 2, k + is, 0)] = o->wtemp2[E2(o, i + is, nj - 5, k + is, 0)];
    else if ((dim == 2) && (k == nk - 1))
      o->wtemp2[E2(o, i + is, j + is, k + 2, 0)] = o->wtemp2[E2(o, i + is, j + is, nk - 5, 0)];
    else if ((dim == 0) && (i == 0))
      o->wtemp2[E2(o, 0, j + is, k + is, 0)] = o->wtemp2[E2(o, 6, j + is, k + is, 0)];
    else if ((dim == 1) && (j == 0))
      o->wtemp2[E2(o, i + is, 0, k + is, 0)] = o->wtemp2[E2(o, i + is, 6, k + is, 0)];
    else if ((dim == 2) && (k == 0))
      o->wtemp2[E2(o, i + is, j + is, 0, 0)] = o->wtemp2[E2(o, i + is, j + is, 6, 0)];
  }
  END_CELLS
}

/* hyperdifvisc2{r,l}: third and first differences on the padded array */
static void k_visc2(O *o, int dim, int right) {
  int a0 = (dim == 0), a1 = (dim == 1), a2 = (dim == 2);
  int kk = (o->nd == 3);
  FOR_CELLS(o)
  int ok = (i > 1 && j > 1 && i < o->n[0] && j < o->n[1]);
  if (o->nd == 3) ok = ok && k > 1 && k < o->n[2];
  if (ok) {
    double *q = o->wtemp2;
    double v;
    if (right)
      v = fabs(3.0 * (q[E2(o, i + a0, j + a1, k + a2 * kk, 0)] - q[E2(o, i, j, k, 0)]) -
               (q[E2(o, i + 2 * a0, j + 2 * a1, k + 2 * a2 * kk, 0)] -
                q[E2(o, i - a0, j - a1, k - a2 * kk, 0)]));
    else
      v = fabs(3.0 * (q[E2(o, i, j, k, 0)] - q[E2(o, i - a0, j - a1, k - a2 * kk, 0)]) -
               (q[E2(o, i + a0, j + a1, k + a2 * kk, 0)] -
                q[E2(o, i - 2 * a0, j - 2 * a1, k - 2 * a2 * kk, 0)]));
    o->wtemp1[E1(o, i, j, k, d3)] = v;
  }
  END_CELLS
  FOR_CELLS(o)
  double *q = o->wtemp2;
  int k1 = k + kk;
  double v;
  if (right)
    v = fabs((q[E2(o, i + a0 + 1, j + a1 + 1, k1 + a2 * kk, 0)] - q[E2(o, i + 1, j + 1, k1, 0)]));
  else
    v = fabs(q[E2(o, i + 1, j + 1, k1, 0)] - (q[E2(o, i - a0 + 1, j - a1 + 1, k1 - a2 * kk, 0)]));
  o->wtemp1[E1(o, i + 1, j + 1, k1, d1)] = v;
  END_CELLS
}

/* hyperdifvisc3{r,l}: local maxima tmp4 (of d3) and tmp5 (of d1) */
static void k_visc3(O *o, int dim) {
  int kk = (o->nd == 3);
  FOR_CELLS(o)
  if (in_interior(o, ii)) {
    int k1 = k + kk;
    double maxt1 = 0, maxt2 = 0;
    for (int s = -1; s <= 1; s++) {
      double v = o->wtemp1[E1(o, i + 1 + s * (dim == 0), j + 1 + s * (dim == 1),
                              k1 + s * (dim == 2) * kk, d3)];
      if (v > maxt1) maxt1 = v;
    }
    o->wtemp[F(o, tmp4) + _c] = maxt1;
    for (int s = -2; s <= 2; s++) {
      double v = o->wtemp1[E1(o, i + 1 + s * (dim == 0), j + 1 + s * (dim == 1),
                              k1 + s * (dim == 2) * kk, d1)];
      if (v > maxt2) maxt2 = v;
    }
    o->wtemp[F(o, tmp5) + _c] = maxt2;
  }
  END_CELLS
}

/* hyperdifvisc4{r,l}: nu = delx*cmax*chyp*tmp4/tmp5 on [2,n-2] */
static void k_visc4(O *o, int field, int dim, int right) {
  FOR_CELLS(o)
  int ok = 1;
  for (int d = 0; d < o->nd; d++)
    if (!(ii[d] > 1 && ii[d] < o->n[d] - 1)) ok = 0;
  if (ok) {
    double *nu = &o->wd[F(o, right ? o->hdnur : o->hdnul) + _c];
    if (o->wtemp[F(o, tmp5) + _c] > 0) {
      double dl = 0;
      for (int d = 0; d < o->nd; d++)
        dl = (d == 0) ? (dim == 0) * (o->wd[F(o, o->delx[0]) + _c])
                      : dl + (dim == d) * (o->wd[F(o, o->delx[d]) + _c]);
      *nu = dl * (o->cmax) * (o->P->chyp[field]) * o->wtemp[F(o, tmp4) + _c] /
            o->wtemp[F(o, tmp5) + _c];
    } else {
      *nu = 0;
    }
  }
  END_CELLS
}

static void hyperdifvisc(O *o, int field, int dim) {
  /* cuhyperdifvisc1ir (src/hyperdifvisc1r.cu:1415-1440) */
  k_visc1(o, field, 1);
  /* cuhyperdifvisc1r (src/hyperdifvisc1r.cu:1303-1413) */
  k_visc1(o, field, 1);
  k_visc1a(o);
  k_visc2(o, dim, 1);
  k_visc3(o, dim);
  k_visc4(o, field, dim, 1);
  /* cuhyperdifvisc1l (src/hyperdifvisc1l.cu:1316-1423) */
  k_visc1(o, field, 0);
  k_visc1a(o);
  k_visc1bcl(o, dim);
  k_visc2(o, dim, 0);
  k_visc3(o, dim);
  k_visc4(o, field, dim, 0);
}

static inline double rdx_of(const O *o, long c, int dim) {
  double r = 0;
  for (int d = 0; d < o->nd; d++)
    r = (d == 0) ? (o->wd[F(o, o->delx[0]) + c]) * (dim == 0)
                 : r + (o->wd[F(o, o->delx[d]) + c]) * (dim == d);
  return r;
}

#define NUR(c) (o->wd[F(o, o->hdnur) + (c)])
#define NUL(c) (o->wd[F(o, o->hdnul) + (c)])
#define NUS(c, dim) (o->wd[F(o, o->nushk[dim]) + (c)])
#define TMP(f, c) (o->wtemp[F(o, f) + (c)])

/* cuhyperdifrhosource1 (src/hyperdifrhosource1.cu:15-275) */
static void k_rhosource(O *o, int field, int dim) {
  FOR_CELLS(o)
  o->dwn1[F(o, field) + _c] = 0.0;
  TMP(tmp1, _c) = 0.0;
  TMP(tmp2, _c) = 0.0;
  END_CELLS
  FOR_CELLS(o)
  if (in_band1(o, ii)) {
    TMP(tmp1, _c) = grad1r3n(o, &o->w0[F(o, o->rho)], ii, dim);
    TMP(tmp2, _c) = grad1l3n(o, &o->w0[F(o, o->rho)], ii, dim);
  }
  END_CELLS
  FOR_CELLS(o)
  double rdx = rdx_of(o, _c, dim);
  double *w = &o->w1[F(o, field) + _c];
  *w = *w + o->dt * ((NUR(_c) + NUS(_c, dim)) * TMP(tmp1, _c) -
                     (NUL(_c) + NUS(_c, dim)) * TMP(tmp2, _c)) / rdx;
  END_CELLS
}

/* cuhyperdifesource1 (src/hyperdifesource1.cu:18-548) */
static void k_esource(O *o, int field, int dim) {
  FOR_CELLS(o)
  for (int f = tmp1; f <= tmp8; f++) TMP(f, _c) = 0.0;
  o->dwn1[F(o, field) + _c] = 0.0;
  END_CELLS
  FOR_CELLS(o)
  TMP(tmp1, _c) = hq(o, o->w0, _c, o->energy);
  END_CELLS
  FOR_CELLS(o)
  if (in_band1(o, ii)) {
    TMP(tmp2, _c) = grad1l3n(o, &o->wtemp[F(o, tmp1)], ii, dim);
    TMP(tmp3, _c) = grad1r3n(o, &o->wtemp[F(o, tmp1)], ii, dim);
  }
  END_CELLS
  FOR_CELLS(o)
  double rdx = rdx_of(o, _c, dim);
  double *w = &o->w1[F(o, field) + _c];
  *w = *w + o->dt * ((NUR(_c) + NUS(_c, dim)) * TMP(tmp3, _c) -
                     (NUL(_c) + NUS(_c, dim)) * TMP(tmp2, _c)) / rdx;
  END_CELLS
}

/* cuhyperdifmomsource1, ii == dim (src/hyperdifmomsource1.cu:17-540) */
static void k_momsource(O *o, int field, int dim, int ii0) {
  const double *w = o->w0;
  int mi = o->mom[ii0];
  FOR_CELLS(o)
  for (int f = tmp1; f <= tmp8; f++) TMP(f, _c) = 0.0;
  o->dwn1[F(o, o->energy) + _c] = 0.0;
  o->dwn1[F(o, mi) + _c] = 0.0;
  END_CELLS
  FOR_CELLS(o)
  TMP(tmp4, _c) = w[F(o, o->mom[field]) + _c] / (w[F(o, o->rho) + _c] + w[F(o, o->rhob) + _c]);
  END_CELLS
  long s = stepd(o, dim);
  FOR_CELLS(o)
  if (in_band1(o, ii)) {
    long c = _c;
    TMP(tmp2, c) = (w[F(o, o->rho) + c] + w[F(o, o->rhob) + c] + w[F(o, o->rho) + c - s] +
                    w[F(o, o->rhob) + c - s]) / 2;
    TMP(tmp3, c) = (w[F(o, o->rho) + c] + w[F(o, o->rhob) + c] + w[F(o, o->rho) + c + s] +
                    w[F(o, o->rhob) + c + s]) / 2;
    TMP(tmp5, c) = (w[F(o, mi) + c] + w[F(o, mi) + c - s]) / 2;
    TMP(tmp6, c) = (w[F(o, mi) + c] + w[F(o, mi) + c + s]) / 2;
  }
  END_CELLS
  FOR_CELLS(o) /* hyperdifmomsource2 */
  if (in_band1(o, ii)) {
    TMP(tmp8, _c) = grad1r3n(o, &o->wtemp[F(o, tmp4)], ii, dim);
    TMP(tmp7, _c) = grad1l3n(o, &o->wtemp[F(o, tmp4)], ii, dim);
  }
  END_CELLS
  FOR_CELLS(o) /* hyperdifmomsource3 */
  double rdx = rdx_of(o, _c, dim);
  o->dwn1[F(o, mi) + _c] = (TMP(tmp3, _c) * (NUR(_c) + NUS(_c, dim)) * TMP(tmp8, _c) -
                            TMP(tmp2, _c) * (NUL(_c) + NUS(_c, dim)) * TMP(tmp7, _c)) /
                           (rdx) / 2;
  o->w1[F(o, mi) + _c] = o->w1[F(o, mi) + _c] + o->dt * o->dwn1[F(o, mi) + _c];
  END_CELLS
  FOR_CELLS(o) /* hyperdifmomsource3a */
  double rdx = rdx_of(o, _c, dim);
  o->dwn1[F(o, o->energy) + _c] =
      (TMP(tmp6, _c) * (NUR(_c) + NUS(_c, dim)) * TMP(tmp8, _c) -
       TMP(tmp5, _c) * (NUL(_c) + NUS(_c, dim)) * TMP(tmp7, _c)) / (rdx) / 2;
  o->w1[F(o, o->energy) + _c] =
      o->w1[F(o, o->energy) + _c] + o->dt * o->dwn1[F(o, o->energy) + _c];
  END_CELLS
}

/* cuhyperdifmomsourcene1, ii != dim (src/hyperdifmomsourcene1.cu:16-745) */
static void k_momsourcene(O *o, int field, int dim, int iix, int ii0) {
  const double *w = o->w0;
  int mi = o->mom[ii0];
  FOR_CELLS(o)
  for (int f = tmp1; f <= tmp8; f++) TMP(f, _c) = 0.0;
  o->dwn1[F(o, o->energy) + _c] = 0.0;
  o->dwn1[F(o, mi) + _c] = 0.0;
  END_CELLS
  FOR_CELLS(o)
  TMP(tmp1, _c) = w[F(o, o->rho) + _c] + w[F(o, o->rhob) + _c];
  TMP(tmp4, _c) = w[F(o, o->mom[field]) + _c] / (w[F(o, o->rho) + _c] + w[F(o, o->rhob) + _c]);
  END_CELLS
  FOR_CELLS(o) /* ne2 */
  if (in_band1(o, ii)) TMP(tmp5, _c) = (grad13n(o, &o->wtemp[F(o, tmp4)], ii, dim));
  END_CELLS
  FOR_CELLS(o) /* ne3 */
  TMP(tmp6, _c) = TMP(tmp5, _c) * ((NUR(_c) + NUL(_c) + 2.0 * NUS(_c, dim))) / 4.0;
  END_CELLS
  FOR_CELLS(o) /* ne4 */
  TMP(tmp7, _c) = TMP(tmp1, _c) * TMP(tmp6, _c);
  TMP(tmp8, _c) = TMP(tmp6, _c) * w[F(o, mi) + _c];
  END_CELLS
  FOR_CELLS(o) /* ne5 */
  o->dwn1[F(o, mi) + _c] = (grad13n(o, &o->wtemp[F(o, tmp7)], ii, iix));
  END_CELLS
  FOR_CELLS(o) /* ne6 */
  o->w1[F(o, mi) + _c] = o->w1[F(o, mi) + _c] + o->dt * o->dwn1[F(o, mi) + _c];
  END_CELLS
  FOR_CELLS(o) /* ne5a */
  if (in_band1(o, ii)) o->dwn1[F(o, o->energy) + _c] = (grad13n(o, &o->wtemp[F(o, tmp8)], ii, iix));
  END_CELLS
  FOR_CELLS(o) /* ne6a */
  o->w1[F(o, o->energy) + _c] =
      o->w1[F(o, o->energy) + _c] + o->dt * o->dwn1[F(o, o->energy) + _c];
  END_CELLS
}

/* cuhyperdifbsource1, mm == dim (src/hyperdifbsource1.cu:21-445) */
static void k_bsource(O *o, int field, int dim, int jj, int ii0, double sb) {
  const double *w = o->w0;
  int bi = o->b[ii0];
  long s = stepd(o, dim);
  FOR_CELLS(o)
  for (int f = tmp1; f <= tmp8; f++) TMP(f, _c) = 0.0;
  o->dwn1[F(o, o->energy) + _c] = 0.0;
  o->dwn1[F(o, bi) + _c] = 0.0;
  END_CELLS
  FOR_CELLS(o)
  if (in_band1(o, ii)) {
    long c = _c;
    TMP(tmp2, c) = (w[F(o, o->b[jj]) + c] + w[F(o, o->b[jj]) + c - s]) / 2;
    TMP(tmp3, c) = (w[F(o, o->b[jj]) + c] + w[F(o, o->b[jj]) + c + s]) / 2;
    TMP(tmp1, c) = w[F(o, o->b[field]) + c];
  }
  END_CELLS
  FOR_CELLS(o) /* bsource2 */
  if (in_band1(o, ii)) {
    TMP(tmp4, _c) = grad1l3n(o, &o->wtemp[F(o, tmp1)], ii, dim);
    TMP(tmp5, _c) = grad1r3n(o, &o->wtemp[F(o, tmp1)], ii, dim);
  }
  END_CELLS
  FOR_CELLS(o) /* bsource3 */
  double rdx = rdx_of(o, _c, dim);
  o->dwn1[F(o, bi) + _c] = sb * (TMP(tmp5, _c) * NUR(_c) - TMP(tmp4, _c) * NUL(_c)) / rdx;
  o->dwn1[F(o, o->energy) + _c] = sb *
                                   (TMP(tmp3, _c) * TMP(tmp5, _c) * NUR(_c) -
                                    TMP(tmp2, _c) * TMP(tmp4, _c) * NUL(_c)) / rdx;
  END_CELLS
  FOR_CELLS(o) /* bsource4 */
  o->w1[F(o, bi) + _c] = o->w1[F(o, bi) + _c] + o->dt * o->dwn1[F(o, bi) + _c];
  o->w1[F(o, o->energy) + _c] =
      o->w1[F(o, o->energy) + _c] + o->dt * o->dwn1[F(o, o->energy) + _c];
  END_CELLS
}

/* cuhyperdifbsourcene1, mm != dim (src/hyperdifbsourcene1.cu:18-825) */
static void k_bsourcene(O *o, int field, int dim, int jj, int ii0, int mm, double sb) {
  const double *w = o->w0;
  int bi = o->b[ii0];
  FOR_CELLS(o)
  for (int f = tmp1; f <= tmp8; f++) TMP(f, _c) = 0.0;
  o->dwn1[F(o, o->energy) + _c] = 0.0;
  o->dwn1[F(o, bi) + _c] = 0.0;
  END_CELLS
  FOR_CELLS(o) /* 1a */
  TMP(tmp1, _c) = w[F(o, o->b[field]) + _c];
  END_CELLS
  FOR_CELLS(o) /* 1b */
  if (in_band1(o, ii)) TMP(tmp2, _c) = grad13n(o, &o->wtemp[F(o, tmp1)], ii, dim);
  END_CELLS
  FOR_CELLS(o) /* 2 */
  TMP(tmp3, _c) = TMP(tmp2, _c) * (NUL(_c) + NUR(_c)) / 2;
  END_CELLS
  FOR_CELLS(o) /* 3 */
  if (in_band1(o, ii)) TMP(tmp4, _c) = grad13n(o, &o->wtemp[F(o, tmp3)], ii, mm);
  END_CELLS
  FOR_CELLS(o) /* 4 */
  TMP(tmp5, _c) = TMP(tmp3, _c) * w[F(o, o->b[jj]) + _c];
  END_CELLS
  FOR_CELLS(o) /* 6 */
  o->dwn1[F(o, bi) + _c] = sb * TMP(tmp4, _c);
  o->w1[F(o, bi) + _c] = o->w1[F(o, bi) + _c] + o->dt * o->dwn1[F(o, bi) + _c];
  END_CELLS
  FOR_CELLS(o) /* 5; the 3D launch bound omits k>0 (src/hyperdifbsourcene1.cu:233) */
  int ok;
  if (o->nd == 3)
    ok = (i > 0 && j > 0 && i < o->n[0] - 1 && j < o->n[1] - 1 && k < o->n[2] - 1);
  else
    ok = in_band1(o, ii);
  if (ok) TMP(tmp6, _c) = grad13n(o, &o->wtemp[F(o, tmp5)], ii, mm);
  END_CELLS
  FOR_CELLS(o) /* 6a */
  o->dwn1[F(o, o->energy) + _c] = sb * TMP(tmp6, _c);
  o->w1[F(o, o->energy) + _c] =
      o->w1[F(o, o->energy) + _c] + o->dt * o->dwn1[F(o, o->energy) + _c];
  END_CELLS
}

/* ---- user source: Gaussian vertical-velocity driver ------------------- */
/* The reference's drivers (models/usersource.cu.spicule1:3-137) add
   m_1 += dt*v*(rho+rhob) with rho read from slot ordero after all other
   updates; v is a product of Gaussians in the cell position.  The time factor
   sin(2 pi t/P) is the reference's commented-out tdep (spicule1:48). */
static double driver_v(const O *o, long c) {
  const smaug_params_t *P = o->P;
  double v = P->drv_amp;
  if (P->drv_period > 0) v *= sin(o->t * 2.0 * M_PI / P->drv_period);
  for (int d = 0; d < o->nd; d++) {
    if (P->drv_sigma[d] > 0) {
      double x = o->wd[F(o, o->pos[d]) + c] - P->drv_x0[d];
      v *= exp(-x * x / (P->drv_sigma[d] * P->drv_sigma[d]));
    }
  }
  return v;
}

/* SMAUG_DRIVER_GAUSS_STEP: the reference's spicule1 model applies its term
   only while p->it == 1 (models/usersource.cu.spicule1:67); p->it is the
   step counter n of the driver loop (src/iosmaug.c:496-498), copied to the
   device by cusource (src/centdiff2.cu:1229) */
static void k_source(O *o) {
  if (o->P->driver == SMAUG_DRIVER_GAUSS_STEP) {
    if (o->it != o->P->drv_step) return;
  } else if (o->P->driver != SMAUG_DRIVER_GAUSS) {
    return;
  }
  FOR_CELLS(o)
  double v = driver_v(o, _c);
  const double *wr = o->increment_mode ? o->w0 : o->w1;
  o->w1[F(o, o->mom[0]) + _c] = o->w1[F(o, o->mom[0]) + _c] +
                                (o->dt) * v * (wr[F(o, o->rho) + _c] + wr[F(o, o->rhob) + _c]);
  END_CELLS
}

/* ---- ghost cells -------------------------------------------------------- */
/* periodic: boundary0/1_parallel (src/boundary.cu:72-225), bc3_periodic1_dir
   (src/gradops.cu:1270-1320); contcd4: models/boundary.cu.fluxtube1:16-85;
   cont/symm/asymm: src/gradops.cu:947-1060,1325-1465 (symm/asymm mirror about
   the face between cells 1 and 2 in 2D, about cell 2 in the 3D branch);
   fixed: the ghost cells are not written (the OT model's cuboundary,
   src/boundary.cu:231-252, dispatches periodic only, and the flux-tube model
   restores type 5 from a store its init sweep never fills,
   models/boundary.cu.fluxtube1:1137-1277), so they keep their initial values.
   Applied per field (rho..b_last) and per dim in the reference's order
   (src/iosmaug.c:830-833). */
static void bc_field_dir(const O *o, double *w, int f, int dir) {
  int n = o->n[dir];
  int type = o->P->boundtype[dir][0];
  long s = stepd(o, dir);
  for (long c = 0; c < o->dimp; c++) {
    int ii[3] = {(int)(c % o->n[0]), (int)((c / o->n[0]) % o->n[1]),
                 (int)(c / ((long)o->n[0] * o->n[1]))};
    int x = ii[dir];
    long base = F(o, f) + c - (long)x * s;
    int src = -1;
    double sgn = 1.0;
    switch (type) {
      case SMAUG_BC_PERIODIC:
        if (x == 0 || x == 1) src = n - 4 + x;
        else if (x == n - 1 || x == n - 2) src = 4 - n + x;
        break;
      case SMAUG_BC_CONTCD4:
        if (x == 0 || x == 1) src = 4 - x;
        else if (x == n - 1) src = n - 5;
        else if (x == n - 2) src = n - 4;
        break;
      case SMAUG_BC_CONT:
        if (x == 0 || x == 1) src = 2;
        else if (x == n - 1 || x == n - 2) src = n - 3;
        break;
      case SMAUG_BC_SYMM:
      case SMAUG_BC_ASYMM:
        if (o->nd == 3) {
          if (x == 0 || x == 1) src = 4 - x;
          else if (x == n - 1 || x == n - 2) src = 2 * n - 6 - x;
        } else {
          if (x == 0 || x == 1) src = 3 - x;
          else if (x == n - 1 || x == n - 2) src = 2 * n - 5 - x;
        }
        if (type == SMAUG_BC_ASYMM) sgn = -1.0;
        break;
      case SMAUG_BC_FIXED:
        break;
      default:
        break;
    }
    if (src >= 0) w[base + (long)x * s] = sgn * w[base + (long)src * s];
  }
}

static void k_boundary(const O *o, double *w) {
  for (int f = o->rho; f <= o->b[o->nd - 1]; f++)
    for (int dir = 0; dir < o->nd; dir++) bc_field_dir(o, w, f, dir);
}

/* ---- one evaluation of the spatial operator ---------------------------- */
/* Runs the rkon==0 step body (src/iosmaug.c:631-835) on slot0 = stage input,
   accumulating into slot1.  cmaxd[dim] must hold the per-dim CFL maxima of
   the stage input.  Boundaries are not applied here. */
static void step_body(O *o, const double *cmaxd) {
  int nd = o->nd;
  for (int dir = 0; dir < nd; dir++) k_computevels(o, dir);
  for (int dir = 0; dir < nd; dir++) {
    for (int f = o->rho; f <= o->mom[nd - 1]; f++) {
      if (f == o->mom[dir]) {
        k_computept(o, dir);
        k_computepbg(o, o->w0);
      }
      k_centdiff1(o, f, dir);
    }
    for (int f = o->energy; f <= o->b[nd - 1]; f++) {
      if (f == o->energy) {
        k_computevels(o, dir);
        k_computepbg(o, o->w0);
        k_computept(o, dir);
      }
      k_centdiff2(o, f, dir);
    }
  }
  k_grav(o);
  if (o->P->hyperdifmom == 1) {
    /* nushk slots stay 0: cunushk1 only runs under USE_SHOCKVISC */
    for (int dim = 0; dim < nd; dim++) {
      o->cmax = cmaxd[dim];
      hyperdifvisc(o, o->rho, dim);
      k_rhosource(o, o->rho, dim);
    }
    for (int dim = 0; dim < nd; dim++) {
      o->cmax = cmaxd[dim];
      hyperdifvisc(o, o->energy, dim);
      k_esource(o, o->energy, dim);
    }
    for (int dim = 0; dim < nd; dim++)
      for (int f = 0; f < nd; f++) {
        o->cmax = cmaxd[dim];
        hyperdifvisc(o, o->mom[f], dim);
        for (int ii1 = 0; ii1 <= 1; ii1++) {
          int iix, ii0;
          if (ii1 == 0) { iix = dim; ii0 = f; }
          else { iix = f; ii0 = dim; }
          if (iix == dim) k_momsource(o, f, dim, ii0);
          else k_momsourcene(o, f, dim, iix, ii0);
        }
      }
    for (int dim = 0; dim < nd; dim++)
      for (int f = 0; f < nd; f++) {
        if (f == dim) continue;
        o->cmax = cmaxd[dim];
        hyperdifvisc(o, o->b[f], dim);
        for (int ii1 = 0; ii1 <= 1; ii1++) {
          int jj, mm, ii0;
          double sb;
          if (ii1 == 0) { jj = dim; mm = f; sb = -1.0; ii0 = dim; }
          else { ii0 = f; mm = dim; sb = 1.0; jj = f; }
          if (mm == dim) k_bsource(o, f, dim, jj, ii0, sb);
          else k_bsourcene(o, f, dim, jj, ii0, mm, sb);
        }
      }
  }
  k_source(o);
}

/* cucomputedervfields at step start (src/computedervfields.cu:1671-1707):
   derived fields vel..pkb zeroed */
static void zero_derived(O *o) {
  FOR_CELLS(o)
  for (int f = o->vel[0]; f <= o->pkb; f++) o->wd[F(o, f) + _c] = 0;
  END_CELLS
}

static void all_cmax(O *o, double *cmaxd) {
  for (int d = 0; d < o->nd; d++) cmaxd[d] = k_cmax(o, d);
}

/* dt rule of src/iosmaug.c:541-616.  Because cucomputec copies the device
   params over the host copy after p->dt=DT (src/computedervfields.cu:2255),
   a rejected CFL candidate leaves the previous step's dt in place. */
static double dt_rule(const O *o, const double *cmaxd, double dt_prev) {
  const smaug_params_t *P = o->P;
  if (P->moddton != 1) return dt_prev;
  double courantmax = SMALLDOUBLE;
  double cm = cmaxd[o->nd - 1];
  for (int d = 0; d < o->nd; d++) {
    double t = cm / P->dx[d];
    if (t > courantmax) courantmax = t;
  }
  double dttemp = P->courant / courantmax;
  if (dttemp > SMALLDOUBLE && dttemp < P->dtmax) return dttemp;
  return dt_prev;
}

static void load_geometry(O *o, const double *pos, const double *delx) {
  for (int d = 0; d < o->nd; d++) {
    memcpy(&o->wd[F(o, o->pos[d])], pos + (long)d * o->dimp, sizeof(double) * o->dimp);
    memcpy(&o->wd[F(o, o->delx[d])], delx + (long)d * o->dimp, sizeof(double) * o->dimp);
  }
}

/* ======================================================================== */
/* Exported API (ctypes)                                                     */
/* ======================================================================== */

/* initgrid (src/init.cu:2502-3060): padded copy of the positions, linear
   extrapolation (1+|ixe-ix|)x_ixe - |ixe-ix| x_ixf into the outer layers
   (dim 0 lower: layers 0..1 from 2,3; other dims lower: 0..2 from 3,4; all
   upper: n-1..n+1 from n-2,n-3, padded indices), pos rewritten from the
   padded copy, delx = (x_{i+1}-x_{i-1})/2. */
int or_grid_metric(int ndim, const int32_t *nn, double *pos, double *delx) {
  int n[3] = {nn[0], nn[1], ndim == 3 ? nn[2] : 1};
  int m[3] = {n[0] + 2, n[1] + 2, ndim == 3 ? n[2] + 2 : 1};
  long dimp = (long)n[0] * n[1] * n[2];
  long msz = (long)m[0] * m[1] * m[2];
  double *T = calloc((size_t)ndim * msz, sizeof(double));
  if (!T) return SMAUG_E_NOMEM;
#define TI(a, b, c, f) (((long)(c) * m[1] + (b)) * m[0] + (a) + (long)(f) * msz)
  int kofs3 = (ndim == 3);
  for (int f = 0; f < ndim; f++)
    for (int c = 0; c < n[2]; c++)
      for (int b = 0; b < n[1]; b++)
        for (int a = 0; a < n[0]; a++)
          T[TI(a + 1, b + 1, c + kofs3, f)] = pos[(long)f * dimp + ((long)c * n[1] + b) * n[0] + a];
  for (int dir = 0; dir < ndim; dir++) {
    for (int layer = 0; layer < 2; layer++) {
      int ixmin, ixmax, ixe, ixf;
      if (layer == 0) { /* upper */
        ixmax = n[dir] + 1; ixmin = n[dir] - 1; ixe = ixmin - 1; ixf = ixe - 1;
      } else {          /* lower */
        ixmin = 0; ixmax = (dir == 0) ? 1 : 2; ixe = ixmax + 1; ixf = ixe + 1;
      }
      for (int f = 0; f < ndim; f++) {
        for (int c = 0; c < m[2]; c++)
          for (int b = 0; b < m[1]; b++)
            for (int a = 0; a < m[0]; a++) {
              int ii[3] = {a, b, c};
              int ix = ii[dir];
              if (ix < ixmin || ix > ixmax) continue;
              int i1[3] = {a, b, c}, i2[3] = {a, b, c};
              i1[dir] = ixe;
              i2[dir] = ixf;
              double w1 = (double)abs(ixe - ix);
              T[TI(a, b, c, f)] = (1 + w1) * T[TI(i1[0], i1[1], i1[2], f)] -
                                  (w1) * T[TI(i2[0], i2[1], i2[2], f)];
            }
      }
    }
  }
  for (int f = 0; f < ndim; f++)
    for (int c = 0; c < n[2]; c++)
      for (int b = 0; b < n[1]; b++)
        for (int a = 0; a < n[0]; a++)
          pos[(long)f * dimp + ((long)c * n[1] + b) * n[0] + a] = T[TI(a + 1, b + 1, c + kofs3, f)];
  for (int dir = 0; dir < ndim; dir++)
    for (int c = 0; c < n[2]; c++)
      for (int b = 0; b < n[1]; b++)
        for (int a = 0; a < n[0]; a++) {
          int p[3] = {a + 1, b + 1, c + kofs3};
          int pp[3] = {p[0], p[1], p[2]}, pm[3] = {p[0], p[1], p[2]};
          pp[dir] += 1;
          pm[dir] -= 1;
          delx[(long)dir * dimp + ((long)c * n[1] + b) * n[0] + a] =
              0.5 * (T[TI(pp[0], pp[1], pp[2], dir)] - T[TI(pm[0], pm[1], pm[2], dir)]);
        }
#undef TI
  free(T);
  return 0;
}

/* Apply the ghost-cell boundaries to a full state array in place. */
int or_boundary(const smaug_params_t *P, double *w) {
  O o;
  int rc = init_O(&o, P);
  if (rc) { free_O(&o); return rc; }
  k_boundary(&o, w);
  free_O(&o);
  return 0;
}

/* Per-dim CFL maxima of a state. */
int or_cmax(const smaug_params_t *P, const double *w, double *cmaxd) {
  O o;
  int rc = init_O(&o, P);
  if (rc) { free_O(&o); return rc; }
  memcpy(o.w0, w, sizeof(double) * o.nvar * o.dimp);
  all_cmax(&o, cmaxd);
  free_O(&o);
  return 0;
}

/*
 * Advance `nsteps` steps.
 *   w      in/out, NVAR*dimp, the reference's slot 1 after boundaries (S_n)
 *   pos,delx geometry from or_grid_metric
 *   state  in/out: [0]=p->dt (previous dt), [1]=t (simulated time),
 *          [2]=the step counter (p->it of the next step)
 *   cmax_out  per-dim CFL maxima of the last step input (may be NULL)
 * integrator: SMAUG_INT_EULER reproduces the reference step; SMAUG_INT_RK4
 * is classical RK4 on the same operator: dt from the CFL maxima of the step
 * input, each stage evaluated with the CFL maxima of its own input.
 */
int or_advance(const smaug_params_t *P, double *w, const double *pos,
               const double *delx, int nsteps, double *state, double *cmax_out) {
  O o;
  int rc = init_O(&o, P);
  if (rc) { free_O(&o); return rc; }
  load_geometry(&o, pos, delx);
  long nw = (long)o.nvar * o.dimp;
  double dtprev = state[0];
  o.t = state[1];
  o.it = (long)state[2];
  double cmaxd[3] = {0, 0, 0};
  double *un = NULL, *acc = NULL, *ustage = NULL, *delta = NULL;
  if (P->integrator == SMAUG_INT_RK4) {
    un = malloc(sizeof(double) * nw);
    acc = malloc(sizeof(double) * nw);
    ustage = malloc(sizeof(double) * nw);
    delta = malloc(sizeof(double) * nw);
    if (!un || !acc || !ustage || !delta) { rc = SMAUG_E_NOMEM; goto out; }
  }
  for (int s = 0; s < nsteps; s++) {
    if (P->integrator == SMAUG_INT_EULER) {
      /* slot0 <- slot1 (cucomputedervfields); slot1 keeps S_n */
      memcpy(o.w0, w, sizeof(double) * nw);
      memcpy(o.w1, w, sizeof(double) * nw);
      zero_derived(&o);
      all_cmax(&o, cmaxd);
      o.dt = dt_rule(&o, cmaxd, dtprev);
      o.increment_mode = 0;
      step_body(&o, cmaxd);
      k_boundary(&o, o.w1);
      memcpy(w, o.w1, sizeof(double) * nw);
      dtprev = o.dt;
      o.t += o.dt;
      o.it++;
    } else {
      static const double cst[4] = {0.5, 0.5, 1.0, 0.0};
      static const double wgt[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
      memcpy(un, w, sizeof(double) * nw);
      memcpy(ustage, w, sizeof(double) * nw);
      memcpy(acc, w, sizeof(double) * nw); /* carries the background fields */
      double t0 = o.t;
      double dt = 0;
      for (int st = 0; st < 4; st++) {
        memcpy(o.w0, ustage, sizeof(double) * nw);
        zero_derived(&o);
        all_cmax(&o, cmaxd);
        if (st == 0) {
          dt = dt_rule(&o, cmaxd, dtprev);
          if (cmax_out) memcpy(cmax_out, cmaxd, sizeof(double) * o.nd);
        }
        o.dt = dt;
        o.t = t0 + (st == 0 ? 0.0 : (st == 3 ? dt : 0.5 * dt));
        /* slot1: zero evolved fields, backgrounds copied (they are read
           from slot ordero by centdiff2ci/addenergyterms) */
        memcpy(o.w1, o.w0, sizeof(double) * nw);
        for (int f = o.rho; f <= o.b[o.nd - 1]; f++)
          memset(&o.w1[F(&o, f)], 0, sizeof(double) * o.dimp);
        o.increment_mode = 1;
        step_body(&o, cmaxd);
        memcpy(delta, o.w1, sizeof(double) * nw);
        for (int f = o.rho; f <= o.b[o.nd - 1]; f++) {
          long b = F(&o, f);
          for (long c = 0; c < o.dimp; c++) {
            double dl = delta[b + c];
            if (st == 0) acc[b + c] = un[b + c] + wgt[0] * dl;
            else if (st < 3) acc[b + c] = acc[b + c] + wgt[st] * dl;
            else acc[b + c] = acc[b + c] + wgt[3] * dl;
            if (st < 3) ustage[b + c] = un[b + c] + cst[st] * dl;
          }
        }
        if (st < 3) k_boundary(&o, ustage);
      }
      k_boundary(&o, acc);
      memcpy(w, acc, sizeof(double) * nw);
      dtprev = dt;
      o.t = t0 + dt;
      o.it++;
      continue;
    }
    if (cmax_out) memcpy(cmax_out, cmaxd, sizeof(double) * o.nd);
  }
  state[0] = dtprev;
  state[1] = o.t;
  state[2] = (double)o.it;
out:
  free(un); free(acc); free(ustage); free(delta);
  free_O(&o);
  return rc;
}

int or_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
