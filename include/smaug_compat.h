/*
 * smaug_compat.h -- the reference's host-wrapper interface served by the
 * B200 engine, so that the reference's own driver (src/iosmaug.c with
 * src/readwrite.c, src/initialisation.c, src/dxroutines.c) links and runs
 * unchanged.
 *
 * The reference declares these wrappers in include/smaugcukernels.h:8-93 and
 * defines them in its .cu files; nvcc compiles those as C++, so the driver
 * (compiled by g++, src/make_inputs:3) references C++-mangled names such as
 *   _Z11cucentdiff1PP6paramsS1_PP5statePPdS6_S6_S6_iidii
 * The mangled name encodes the struct tags `params`, `state` and `bparams`
 * and real=double, so this header declares structs with those tags, and the
 * functions below have exactly the reference's parameter types.  The struct
 * layouts must equal the reference's include/iotypes.h:85-190 and
 * include/iobparams.h:9-30 for the same build macros: the driver allocates and
 * fills `struct params` and passes it by pointer.  Supported macro sets:
 *   -DUSE_SAC     2D, NVAR 10   (libsmaug_compat2d.so)
 *   -DUSE_SAC_3D  3D, NVAR 13   (libsmaug_compat3d.so)
 * with real=double and neither USE_MULTIGPU nor ADIABHYDRO.
 *
 * Call protocol.  The shim runs the engine's fused step once per driver
 * iteration instead of one kernel group per wrapper.  This is exact for the
 * single-step (rkon=0) iteration of src/iosmaug.c:496-835 and its output
 * calls (:509-523, :1107):
 *   cucomputedervfields  start of a step: no device work
 *   cucomputec           first call of a step: captures the driver's DT from
 *                        p->dt and, as the reference's params copy-back
 *                        (src/computedervfields.cu:2255) does, leaves the
 *                        previous step's dt in p->dt
 *   cucomputemaxc        p->cmax = CFL maximum of the current state along dir
 *   cucomputevels, cucomputept, cucomputepbg, cucentdiff1, cucentdiff2, cugrav,
 *   cuhyperdifvisc1ir/1r/1l, cuhyperdif*source1   no device work
 *   cusource             runs the whole step (fluxes, hyperdiffusion, source,
 *                        ghost images) with the engine's dt, which must equal
 *                        the dt argument
 *   cuboundary           no device work (the step wrote the ghost layers)
 *   cuupdate             every cfgsavefrequency steps, host wmod slot 0 gets
 *                        the state before the step and slot 1 the state after
 *                        it, as the reference's copy of device slots 0-1
 *                        (src/update.cu:207) does
 * Unsupported: rkon=1 (the reference's RK driver), divbon=1, shock viscosity,
 * fields of one dimension with different boundary types, boundary types
 * other than periodic (0), contcd4 (4) and fixed (5: the ghost layers keep
 * their initial values, as in the OT model build, whose cuboundary dispatches
 * periodic only, src/boundary.cu:231-252); cont, symm and asymm are left out
 * because no model's cuboundary dispatches them, so their meaning depends on
 * the model file.  The reference's wrappers report no errors and the driver
 * ignores their return values, so an unsupported use or an engine error is
 * printed to stderr and ends the process with status 3.
 *
 * The reference's user source terms (src/usersource.cu, models/usersource.*)
 * are compile-time code; the shim's source term is the engine's built-in
 * Gaussian driver, off unless set by smaug_compat_set_driver or the
 * SMAUG_COMPAT_DRIVER environment variable (below).  SMAUG_COMPAT_PRECISION=mixed
 * selects the engine's mixed precision form.
 */
#ifndef SMAUG_COMPAT_H_
#define SMAUG_COMPAT_H_

#include "smaug_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Engine source term used by the shim: m_0 += dt * v * rho_t with
   v = amp * sin(2 pi t / period) * prod_d exp(-((x_d - x0_d) / sigma_d)^2).
   Call before the driver's first step.  The environment variable
   SMAUG_COMPAT_DRIVER="amp,period,x0_0,x0_1,x0_2,sigma_0,sigma_1,sigma_2"
   does the same for an unchanged driver.  No counterpart in the reference. */
int smaug_compat_set_driver(double amp, double period, const double* x0, const double* sigma);

/* The engine handle behind the shim (NULL before the first step), for use of
   the primary ABI alongside the driver.  No counterpart in the reference. */
smaug_handle_t smaug_compat_handle(void);

#ifdef __cplusplus
}
#endif

#ifdef __cplusplus

#if defined(USE_SAC_3D)
#define SMAUG_COMPAT_NDIM 3
#define SMAUG_COMPAT_NVAR 13
#else
#define SMAUG_COMPAT_NDIM 2
#define SMAUG_COMPAT_NVAR 10
#endif

/* include/iotypes.h:85-175 for real=double, without USE_MULTIGPU/ADIABHYDRO */
struct params {
  int n[SMAUG_COMPAT_NDIM];
  int ng[SMAUG_COMPAT_NDIM];
  int npgp[SMAUG_COMPAT_NDIM];
  int fullgridini;
  double hdmean, hdmax, pmax, pmin, pmean, emax, emin, emean;
  double xmax[SMAUG_COMPAT_NDIM];
  double xmin[SMAUG_COMPAT_NDIM];
  int nt;
  int it;
  double tmax;
  double qt;
  double boundu[SMAUG_COMPAT_NDIM][SMAUG_COMPAT_NVAR];
  double boundl[SMAUG_COMPAT_NDIM][SMAUG_COMPAT_NVAR];
  double cmax;
  double maxcourant;
  int steeringenabled;
  int finishsteering;
  double dt;
  double dx[SMAUG_COMPAT_NDIM];
  double gamma;
  double mu;
  double eta;
  double g[SMAUG_COMPAT_NDIM];
  int sodifon, rkon, moddton, divbon, divbfix, cfgsavefrequency, hyperdifmom, mode, readini;
  double courant;
  double maxviscoef;
  double dtdiffvisc;
  double chyp[SMAUG_COMPAT_NVAR];
  double chyp3;
  double test;
  int boundtype[SMAUG_COMPAT_NVAR][SMAUG_COMPAT_NDIM][2];
  int gpid[16];
  int npe;
  int noghost;
};

/* include/iotypes.h:178-190 */
struct state {
  int it;
  double t, dt, rho, m1, m2, m3, e, b1, b2, b3;
};

/* include/iobparams.h:9-30 (fixed-boundary store, MSIZE 128) */
struct bparams {
#if SMAUG_COMPAT_NDIM == 3
  double fixed1[4 * 128 * 128 * SMAUG_COMPAT_NVAR];
  double fixed2[4 * 128 * 128 * SMAUG_COMPAT_NVAR];
  double fixed3[4 * 128 * 128 * SMAUG_COMPAT_NVAR];
#else
  double fixed1[4 * 128 * SMAUG_COMPAT_NVAR];
  double fixed2[4 * 128 * SMAUG_COMPAT_NVAR];
#endif
};

/* include/smaugcukernels.h:8-93; each replaces the wrapper of the same name */
int cuinit(params** p, bparams** bp, double** wmod, double** wnew, double** wd, state** st,
           params** d_p, bparams** d_bp, double** d_wnew, double** d_wmod, double** d_dwn1,
           double** d_wd, state** d_state, double** d_wtemp, double** d_wtemp1, double** d_wtemp2);
int cuupdatemod(params** p, bparams** bp, double** w, double** wnew, double** wd, state** st,
                params** d_p, bparams** d_bp, double** d_w, double** d_wnew, double** d_wmod,
                double** d_dwn1, double** d_wd, state** d_state, double** d_wtemp,
                double** d_wtemp1, double** d_wtemp2);
int initgrid(params** p, state** st, double** wd, params** d_p, double** d_dwn1, double** d_wd,
             state** d_state, double** d_wtemp, double** d_wtemp1, double** d_wtemp2);
int cufinish(params** p, double** w, double** wnew, state** st, params** d_p, bparams** d_bp,
             double** d_w, double** d_wnew, double** d_wmod, double** d_dwn1, double** d_wd,
             state** d_state, double** d_wtemp, double** d_wtemp1, double** d_wtemp2);
int cuboundary(params** p, bparams** bp, params** d_p, bparams** d_bp, state** d_s,
               double** d_wmod, int order, int idir, int field);
int cuupdate(params** p, double** w, double** wmod, double** wtemp2, state** st, params** d_p,
             double** d_w, double** d_wmod, double** d_wtemp2, state** d_state, int step);
int cuupdatehostwd(params** p, double** wd, double** wmod, double** wtemp2, state** st,
                   params** d_p, double** d_wd, double** d_wmod, double** d_wtemp2,
                   state** d_state, int step);
int cuupdatedevicewd(params** p, double** wd, double** wmod, double** wtemp2, state** st,
                     params** d_p, double** d_wd, double** d_wmod, double** d_wtemp2,
                     state** d_state, int step);
int cucentdiff1(params** p, params** d_p, state** d_s, double** d_w, double** d_wmod,
                double** d_dwn1, double** d_wd, int order, int ordero, double dt, int field,
                int dir);
int cucentdiff2(params** p, params** d_p, state** d_s, double** d_w, double** d_wmod,
                double** d_dwn1, double** d_wd, int order, int ordero, double dt, int field,
                int dir);
int cugrav(params** p, params** d_p, state** d_s, double** d_w, double** d_wmod, double** d_dwn1,
           double** d_wd, int order, int ordero, double dt);
int cusource(params** p, params** d_p, state** d_s, double** d_w, double** d_wmod,
             double** d_dwn1, double** d_wd, int order, int ordero, double dt);
int cuadvance(params** p, params** d_p, double** d_wmod, double** d_w, int order);
int cucomputedervfields(params** p, params** d_p, double** d_wmod, double** d_wd, int order);
int cucomputevels(params** p, params** d_p, double** d_wmod, double** d_wd, int order, int dir);
int cucomputemaxc(params** p, params** d_p, double** d_wmod, double** d_wd, int order, int dir,
                  double** wd, double** d_wtemp);
int cucomputemaxcourant(params** p, params** d_p, double** d_wmod, double** d_wd, int order,
                        int dir, double** wd, double** d_wtemp);
int cucomputec(params** p, params** d_p, double** d_wmod, double** d_wd, int order, int dir);
int cucomputept(params** p, params** d_p, double** d_wmod, double** d_wd, int order, int dir);
int cucomputepk(params** p, params** d_p, double** d_wmod, double** d_wd, int order, int dir);
int cucomputepbg(params** p, params** d_p, double** d_wmod, double** d_wd, int order, int dir);
int cudivb(params** p, params** d_p, double** d_w, double** d_wmod, double** d_dwn1,
           double** d_wd, int order, int ordero, double dt);
int cuhyperdifmomsource1(params** p, params** d_p, double** d_wmod, double** d_dwn1,
                         double** d_wd, int order, int ordero, double** d_wtemp, int field,
                         int dim, int ii, int ii0, double dt);
int cuhyperdifmomsourcene1(params** p, params** d_p, double** d_wmod, double** d_dwn1,
                           double** d_wd, int order, int ordero, double** d_wtemp, int field,
                           int dim, int ii, int ii0, double dt);
int cuhyperdifesource1(params** p, params** d_p, double** d_wmod, double** d_dwn1, double** d_wd,
                       int order, int ordero, double** d_wtemp, int field, int dim, double dt);
int cuhyperdifbsource1(params** p, params** d_p, double** d_wmod, double** d_dwn1, double** d_wd,
                       int order, int ordero, double** d_wtemp, int field, int dim, int jj,
                       int ii0, int mm, double sb, double dt);
int cuhyperdifbsourcene1(params** p, params** d_p, double** d_wmod, double** d_dwn1,
                         double** d_wd, int order, int ordero, double** d_wtemp, int field,
                         int dim, int jj, int ii0, int mm, double sb, double dt);
int cuhyperdifrhosource1(params** p, params** d_p, double** d_wmod, double** d_dwn1,
                         double** d_wd, int order, int ordero, double** d_wtemp, int field,
                         int dim, double dt);
int cunushk1(params** p, params** d_p, double** d_wmod, double** d_wd, int order,
             double** d_wtemp, double** d_wtemp1, double** d_wtemp2);
int cugetdtvisc1(params** p, params** d_p, double** d_wmod, double** wd, double** d_wd, int order,
                 double** d_wtemp, double** d_wtemp1, double** d_wtemp2);
int cuhyperdifvisc1(params** p, params** d_p, double** d_wmod, double** d_wd, int order,
                    double** d_wtemp, double** d_wtemp1, double** d_wtemp2, int field, int dim,
                    int hand);
int cuhyperdifvisc1r(params** p, params** d_p, double** d_wmod, double** wd, double** d_wd,
                     int order, double** d_wtemp, double** d_wtemp1, double** d_wtemp2, int field,
                     int dim);
int cuhyperdifvisc1l(params** p, params** d_p, double** d_wmod, double** wd, double** d_wd,
                     int order, double** d_wtemp, double** d_wtemp1, double** d_wtemp2, int field,
                     int dim);
int cuhyperdifvisc1ir(params** p, params** d_p, double** d_wmod, double** d_wd, int order,
                      double** d_wtemp, double** d_wtemp1, double** d_wtemp2, int field, int dim);
int cuhyperdifvisc1il(params** p, params** d_p, double** d_wmod, double** d_wd, int order,
                      double** d_wtemp, double** d_wtemp1, double** d_wtemp2, int field, int dim);
int cuhyperdifviscmax(params** p, double** w, double** wnew, params** d_p, double** d_w,
                      double** d_wnew, double** d_wmod, double** d_dwn1, double** d_wd, int order,
                      double** d_wtemp, int field, int dim);
int cusync(params** p);

#endif /* __cplusplus */

#endif /* SMAUG_COMPAT_H_ */
