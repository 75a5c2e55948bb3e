// compat.cpp -- the reference's host wrappers (include/smaugcukernels.h:8-93)
// implemented on the engine's C ABI, so that the reference driver
// src/iosmaug.c links against this library unchanged.
//
// Built twice, with -DUSE_SAC (2D) and -DUSE_SAC_3D (3D), as the reference is:
// the layout of `struct params` depends on NDIM and NVAR.  One engine per
// process, as the reference keeps one run per process.  The protocol (which
// call runs the step, which calls only update host-visible values) is stated
// in include/smaug_compat.h.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "smaug_compat.h"

namespace {

constexpr int ND = SMAUG_COMPAT_NDIM;
constexpr int NV = SMAUG_COMPAT_NVAR;
// derived-field slots of wd (include/iotypes.h:219-226): pos1.. and delx1..
constexpr int WD_POS = (ND == 3) ? 17 : 15;
constexpr int WD_DELX = (ND == 3) ? 20 : 17;

struct Shim {
  smaug_handle_t h = nullptr;
  long ncell = 0;
  std::vector<double> w0;      // slot 0 of wmod as given to cuinit
  std::vector<double> pos0;    // positions as given to cuinit (before initgrid)
  std::vector<double> before;  // state before the step in flight (for cuupdate)
  bool have_before = false;
  state st0{};                 // *state at cuinit: the reference's device copy
  double dt0 = 0.0;            // p->dt at cuinit (the first step's fallback dt)
  bool started = false;        // cuinit done
  bool in_step = false;        // between cucomputedervfields and cusource
  bool dt_fixed = false;       // p->dt already reset for this step
  bool drv_set = false;
  double drv[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // amp, period, x0[3], sigma[3]
};
Shim S;

[[noreturn]] void die(const char* fn, const char* msg) {
  std::fprintf(stderr, "smaug_compat: %s: %s\n", fn, msg);
  std::fflush(stderr);
  std::exit(3);
}

void check(const char* fn, int rc) {
  if (rc) die(fn, smaug_last_error());
}

void need_started(const char* fn) {
  if (!S.started) die(fn, "called before cuinit");
}

void read_env_driver() {
  const char* s = std::getenv("SMAUG_COMPAT_DRIVER");
  if (!s || S.drv_set) return;
  double v[8];
  int k = 0;
  const char* c = s;
  while (k < 8) {
    char* end = nullptr;
    v[k] = std::strtod(c, &end);
    if (end == c) break;
    k++;
    c = end;
    if (*c == ',') c++;
  }
  if (k != 8) die("cuinit", "SMAUG_COMPAT_DRIVER needs 8 comma-separated numbers");
  std::memcpy(S.drv, v, sizeof(v));
  S.drv_set = true;
}

// Create the engine from the state and positions given to cuinit.  dtmax is
// the driver's DT (p->dt as the driver resets it before the first CFL call
// of a step, src/iosmaug.c:545-546).
void create_engine(const params* p, double dtmax) {
  smaug_params_t ep;
  check("cuinit", smaug_params_default(&ep, ND));
  for (int d = 0; d < 3; d++) ep.n[d] = d < ND ? p->n[d] : 1;
  ep.moddton = p->moddton == 1 ? 1 : 0;
  ep.hyperdifmom = p->hyperdifmom == 1 ? 1 : 0;
  ep.integrator = SMAUG_INT_EULER;
  ep.precision = SMAUG_PREC_FP64;
  const char* prec = std::getenv("SMAUG_COMPAT_PRECISION");
  if (prec && !std::strcmp(prec, "mixed")) ep.precision = SMAUG_PREC_MIXED;
  ep.pad_model = SMAUG_PAD_STRAY;
#ifdef USE_DORDER3
  ep.stencil_order = 6;  // the reference's 6th-order grad3dn build (src/gradops.cu:450-453)
#endif
  for (int d = 0; d < ND; d++)
    for (int s = 0; s < 2; s++) {
      for (int f = 1; f < NV; f++)
        if (p->boundtype[f][d][s] != p->boundtype[0][d][s])
          die("cuinit", "fields of one dimension with different boundary types");
      ep.boundtype[d][s] = p->boundtype[0][d][s];
    }
  for (int d = 0; d < 3; d++) {
    ep.dx[d] = d < ND ? p->dx[d] : 0.0;
    ep.g[d] = d < ND ? p->g[d] : 0.0;
    ep.xmin[d] = d < ND ? p->xmin[d] : 0.0;
  }
  ep.dt = S.dt0;
  ep.dtmax = dtmax;
  ep.courant = p->courant;
  ep.gamma = p->gamma;
  ep.eta = p->eta;
  for (int f = 0; f < NV; f++) ep.chyp[f] = p->chyp[f];
  if (S.drv_set && S.drv[0] != 0.0) {
    ep.driver = SMAUG_DRIVER_GAUSS;
    ep.drv_amp = S.drv[0];
    ep.drv_period = S.drv[1];
    for (int d = 0; d < 3; d++) {
      ep.drv_x0[d] = S.drv[2 + d];
      ep.drv_sigma[d] = S.drv[5 + d];
    }
  }
  check("cuinit", smaug_create(&ep, S.w0.data(), S.pos0.data(), &S.h));
  S.w0.clear();
  S.w0.shrink_to_fit();
}

void ensure_engine(const char* fn, const params* p) {
  if (S.h) return;
  if (p->moddton == 1) die(fn, "first step did not start with cucomputec (src/iosmaug.c:541-553)");
  create_engine(p, p->dt);
}

double engine_dt(const char* fn) {
  double dt = 0.0;
  check(fn, smaug_get_time(S.h, nullptr, nullptr, &dt));
  return dt;
}

}  // namespace

// ---------------------------------------------------------------------------
// extras (no counterpart in the reference)
// ---------------------------------------------------------------------------
extern "C" int smaug_compat_set_driver(double amp, double period, const double* x0,
                                       const double* sigma) {
  if (S.h) return SMAUG_E_INVALID;  // the engine already runs
  S.drv[0] = amp;
  S.drv[1] = period;
  for (int d = 0; d < 3; d++) {
    S.drv[2 + d] = x0 ? x0[d] : 0.0;
    S.drv[5 + d] = sigma ? sigma[d] : 0.0;
  }
  S.drv_set = true;
  return SMAUG_OK;
}

extern "C" smaug_handle_t smaug_compat_handle(void) { return S.h; }

// ---------------------------------------------------------------------------
// set-up and output (src/init.cu:2222-2448, :2502-3060, src/update.cu:165-233)
// ---------------------------------------------------------------------------
int cuinit(params** p, bparams**, double** wmod, double**, double** wd, state** st, params**,
           bparams**, double**, double**, double**, double**, state**, double**, double**,
           double**) {
  if (S.started) die("cuinit", "called twice (one engine per process)");
  const params* P = *p;
  if (P->rkon != 0) die("cuinit", "rkon=1 (the reference's RK driver) is not supported");
  long nc = 1;
  for (int d = 0; d < ND; d++) {
    if (P->n[d] < 8) die("cuinit", "fewer than 8 cells along a dimension");
    nc *= P->n[d];
  }
  S.ncell = nc;
  S.w0.assign(*wmod, *wmod + (size_t)NV * nc);
  S.pos0.assign(*wd + (size_t)WD_POS * nc, *wd + (size_t)(WD_POS + ND) * nc);
  S.st0 = **st;
  S.dt0 = P->dt;
  read_env_driver();
  S.started = true;
  return 0;
}

int initgrid(params** p, state**, double** wd, params**, double**, double**, state**, double**,
             double**, double**) {
  need_started("initgrid");
  int32_t n[3] = {1, 1, 1};
  for (int d = 0; d < ND; d++) n[d] = (*p)->n[d];
  // the reference rewrites the host copy of the positions and cell widths
  check("initgrid", smaug_grid_metric(ND, n, *wd + (size_t)WD_POS * S.ncell,
                                      *wd + (size_t)WD_DELX * S.ncell));
  return 0;
}

int cuboundary(params** p, bparams**, params**, bparams**, state**, double**, int, int idir,
               int field) {
  need_started("cuboundary");
  // types whose meaning does not depend on the model's boundary.cu: periodic,
  // contcd4 and fixed (ghosts keep their initial values)
  for (int side = 0; side < 2; side++) {
    const int t = (*p)->boundtype[field][idir][side];
    if (t != SMAUG_BC_PERIODIC && t != SMAUG_BC_CONTCD4 && t != SMAUG_BC_FIXED)
      die("cuboundary", "boundary type other than periodic (0), contcd4 (4) or fixed (5)");
  }
  return 0;  // the engine's step writes the ghost layers
}

int cuupdate(params** p, double**, double** wmod, double**, state** st, params**, double**,
             double**, double**, state**, int step) {
  need_started("cuupdate");
  const int freq = (*p)->cfgsavefrequency;
  if (freq > 0 && step % freq == 0 && S.h) {
    const size_t slot = (size_t)NV * S.ncell;
    if (S.have_before)
      std::memcpy(*wmod, S.before.data(), slot * sizeof(double));
    else
      check("cuupdate", smaug_get_state(S.h, *wmod));
    check("cuupdate", smaug_get_state(S.h, *wmod + slot));
    **st = S.st0;
  }
  S.have_before = false;
  return 0;
}

int cusync(params**) {
  if (S.h) check("cusync", smaug_sync(S.h));
  return 0;
}

int cufinish(params**, double**, double**, state**, params**, bparams**, double**, double**,
             double**, double**, double**, state**, double**, double**, double**) {
  if (S.h) check("cufinish", smaug_destroy(S.h));
  S.h = nullptr;
  return 0;
}

// ---------------------------------------------------------------------------
// the single-step iteration (src/iosmaug.c:496-835)
// ---------------------------------------------------------------------------
int cucomputedervfields(params** p, params**, double**, double**, int) {
  need_started("cucomputedervfields");
  if ((*p)->rkon != 0) die("cucomputedervfields", "rkon=1 is not supported");
  S.in_step = true;
  S.dt_fixed = false;
  return 0;
}

int cucomputec(params** p, params**, double**, double**, int, int) {
  need_started("cucomputec");
  params* P = *p;
  if (!S.h) {
    if (!S.in_step) die("cucomputec", "called outside a step");
    create_engine(P, P->dt);  // p->dt holds the driver's DT here
  }
  if (S.in_step && !S.dt_fixed && P->moddton == 1) {
    // the reference copies the device params over the host ones here
    // (src/computedervfields.cu:2255): p->dt becomes the previous step's dt
    P->dt = engine_dt("cucomputec");
    S.dt_fixed = true;
  }
  return 0;
}

int cucomputemaxc(params** p, params**, double**, double**, int, int dir, double**, double**) {
  need_started("cucomputemaxc");
  ensure_engine("cucomputemaxc", *p);
  if (dir < 0 || dir >= ND) die("cucomputemaxc", "dir out of range");
  double c[3] = {0, 0, 0};
  check("cucomputemaxc", smaug_get_cmax(S.h, c));
  (*p)->cmax = c[dir];
  return 0;
}

int cusource(params** p, params**, state**, double**, double**, double**, double**, int, int,
             double dt) {
  need_started("cusource");
  ensure_engine("cusource", *p);
  const int freq = (*p)->cfgsavefrequency;
  S.have_before = false;
  if (freq > 0 && (*p)->it % freq == 0) {
    S.before.resize((size_t)NV * S.ncell);
    check("cusource", smaug_get_state(S.h, S.before.data()));
    S.have_before = true;
  }
  check("cusource", smaug_step(S.h, 1));
  const double de = engine_dt("cusource");
  if (!(std::fabs(de - dt) <= 1e-13 * std::fabs(dt))) {
    char msg[200];
    std::snprintf(msg, sizeof(msg),
                  "driver dt %.17g differs from the engine's %.17g (call sequence is not "
                  "src/iosmaug.c's single-step iteration)", dt, de);
    die("cusource", msg);
  }
  S.in_step = false;
  return 0;
}

// terms computed inside the engine's step
int cucomputevels(params**, params**, double**, double**, int, int) { return 0; }
int cucomputept(params**, params**, double**, double**, int, int) { return 0; }
int cucomputepk(params**, params**, double**, double**, int, int) { return 0; }
int cucomputepbg(params**, params**, double**, double**, int, int) { return 0; }
int cucentdiff1(params**, params**, state**, double**, double**, double**, double**, int, int,
                double, int, int) {
  return 0;
}
int cucentdiff2(params**, params**, state**, double**, double**, double**, double**, int, int,
                double, int, int) {
  return 0;
}
int cugrav(params**, params**, state**, double**, double**, double**, double**, int, int, double) {
  return 0;
}
int cuhyperdifvisc1ir(params**, params**, double**, double**, int, double**, double**, double**,
                      int, int) {
  return 0;
}
int cuhyperdifvisc1il(params**, params**, double**, double**, int, double**, double**, double**,
                      int, int) {
  return 0;
}
int cuhyperdifvisc1r(params**, params**, double**, double**, double**, int, double**, double**,
                     double**, int, int) {
  return 0;
}
int cuhyperdifvisc1l(params**, params**, double**, double**, double**, int, double**, double**,
                     double**, int, int) {
  return 0;
}
int cuhyperdifrhosource1(params**, params**, double**, double**, double**, int, int, double**,
                         int, int, double) {
  return 0;
}
int cuhyperdifesource1(params**, params**, double**, double**, double**, int, int, double**, int,
                       int, double) {
  return 0;
}
int cuhyperdifmomsource1(params**, params**, double**, double**, double**, int, int, double**,
                         int, int, int, int, double) {
  return 0;
}
int cuhyperdifmomsourcene1(params**, params**, double**, double**, double**, int, int, double**,
                           int, int, int, int, double) {
  return 0;
}
int cuhyperdifbsource1(params**, params**, double**, double**, double**, int, int, double**, int,
                       int, int, int, int, double, double) {
  return 0;
}
int cuhyperdifbsourcene1(params**, params**, double**, double**, double**, int, int, double**,
                         int, int, int, int, int, double, double) {
  return 0;
}

// ---------------------------------------------------------------------------
// not reached by the single-GPU single-step driver
// ---------------------------------------------------------------------------
int cudivb(params**, params**, double**, double**, double**, double**, int, int, double) {
  die("cudivb", "divbon=1 is not supported");
}
int cuadvance(params**, params**, double**, double**, int) {
  die("cuadvance", "the reference's RK driver (rkon=1) is not supported");
}
int cunushk1(params**, params**, double**, double**, int, double**, double**, double**) {
  die("cunushk1", "shock viscosity is not supported (the reference never assigns it, "
                  "src/nushk1.cu:346-349)");
}
int cuupdatemod(params**, bparams**, double**, double**, double**, state**, params**, bparams**,
                double**, double**, double**, double**, double**, state**, double**, double**,
                double**) {
  die("cuupdatemod", "not supported");
}
int cuupdatehostwd(params**, double**, double**, double**, state**, params**, double**, double**,
                   double**, state**, int) {
  die("cuupdatehostwd", "derived fields are not kept on the device");
}
int cuupdatedevicewd(params**, double**, double**, double**, state**, params**, double**,
                     double**, double**, state**, int) {
  die("cuupdatedevicewd", "derived fields are not kept on the device");
}
int cucomputemaxcourant(params**, params**, double**, double**, int, int, double**, double**) {
  die("cucomputemaxcourant", "not supported");
}
int cugetdtvisc1(params**, params**, double**, double**, double**, int, double**, double**,
                 double**) {
  die("cugetdtvisc1", "not supported");
}
int cuhyperdifvisc1(params**, params**, double**, double**, int, double**, double**, double**, int,
                    int, int) {
  die("cuhyperdifvisc1", "not supported");
}
int cuhyperdifviscmax(params**, double**, double**, params**, double**, double**, double**,
                      double**, double**, int, double**, int, int) {
  die("cuhyperdifviscmax", "not supported");
}
