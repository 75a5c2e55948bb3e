/*
 * smaug_b200.h -- C ABI of the B200-native SMAUG time-advance engine.
 *
 * The engine replaces the single-GPU time-advance path of SMAUG (Sheffield
 * MHD code, mikeg64/smaug): the host wrappers declared in the reference's
 * include/smaugcukernels.h:8-93 and driven once per step by
 * src/iosmaug.c:496-1144.  The reference calls ~40 wrappers per step, each
 * launching 1-9 kernels with a host synchronisation after every launch; this
 * library advances whole steps with a few fused kernels per step.
 *
 * Conventions (all unchanged from the reference):
 *   - State layout: structure of arrays, field-major, x fastest:
 *       w[f*n0*n1*n2 + (k*n1 + j)*n0 + i]            (src/gradops.cu:44-54)
 *     field order 2D: rho mom1 mom2 energy b1 b2 energyb rhob b1b b2b
 *                 3D: rho mom1 mom2 mom3 energy b1 b2 b3 energyb rhob b1b b2b b3b
 *     (include/iotypes.h:209-216).  n[d] includes 2 ghost layers on each side.
 *   - Positions: pos[d*n0*n1*n2 + cell] as read from the .ini file
 *     (src/readwrite.c:1061-1068); the grid metric delx is derived from them
 *     exactly as initgrid does (src/init.cu:2502-3060).
 *   - Arithmetic: FP64 (the reference's real=double, include/iotypes.h:8-12).
 *
 * Every entry point returns 0 on success and a nonzero SMAUG_E* code on
 * failure; smaug_last_error() returns a message for the calling thread's last
 * failure.  A handle is owned by one host thread at a time; different handles
 * are independent.
 */
#ifndef SMAUG_B200_H_
#define SMAUG_B200_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SMAUG_PARAMS_VERSION 1
#define SMAUG_MAXVAR 13

/* status codes */
#define SMAUG_OK 0
#define SMAUG_E_INVALID 1      /* bad argument or parameter block */
#define SMAUG_E_CUDA 2         /* CUDA runtime error (message has the CUDA string) */
#define SMAUG_E_NOMEM 3        /* device or host allocation failed */
#define SMAUG_E_IO 4           /* file could not be read or written */
#define SMAUG_E_FORMAT 5       /* malformed .ini/.out content */
#define SMAUG_E_UNSUPPORTED 6  /* valid in the reference, not implemented here */
#define SMAUG_E_NONFINITE 7    /* a NaN/Inf appeared in the evolved state */

/* boundary types, numbering of p->boundtype (include/iotypes.h:139) */
#define SMAUG_BC_PERIODIC 0
#define SMAUG_BC_CONT 3
#define SMAUG_BC_CONTCD4 4
#define SMAUG_BC_FIXED 5
#define SMAUG_BC_SYMM 6
#define SMAUG_BC_ASYMM 7

/* integrators */
#define SMAUG_INT_EULER 0  /* the reference's rkon=0 single-stage step */
#define SMAUG_INT_RK4 1    /* classical RK4 on the same spatial operator */

/* precision forms */
#define SMAUG_PREC_FP64 0
/* mixed: perturbation fields stored in float (the base state as a float
   high/low pair), backgrounds, fluxes, pressure recovery, CFL speeds and the
   RK4 accumulator in double, hyperdiffusion arithmetic in float; the host
   interface (get/set state, .out files) stays FP64 */
#define SMAUG_PREC_MIXED 1

/* Fill model of the outer layer of the padded array from which the
   reference's right-biased hyperviscosity is computed.  hyperdifvisc1r_parallel
   (src/hyperdifvisc1r.cu:1099-1258) zeroes that array and, in the same
   launch, stores tmp6 through encode3 instead of encode3p2; the stray stores
   that land in the pad race with the zeroing.  Inside a 512-thread block the
   stray store lands last, which is what the reference produced on a B200. */
#define SMAUG_PAD_STRAY 0  /* pad holds the stray tmp6 store */
#define SMAUG_PAD_ZERO 1   /* pad holds zero */

/* user source (driver) kinds */
#define SMAUG_DRIVER_NONE 0
#define SMAUG_DRIVER_GAUSS 1  /* m_0 += dt * v(x,t) * rho_t, v Gaussian in space */
/* the same term in one step only: the step whose counter (the reference's
   p->it = n, src/iosmaug.c:498) equals drv_step -- the reference's spicule1
   model kicks at p->it == 1 only (models/usersource.cu.spicule1:67-131) */
#define SMAUG_DRIVER_GAUSS_STEP 2

/*
 * Run parameters.  Mirrors the fields of the reference's struct params
 * (include/iotypes.h:85-175) that the time advance reads; the per-field
 * boundtype[NVAR][NDIM][2] is given per dimension because the reference
 * driver assigns the same type to every field (src/iosmaug.c:192-222).
 */
typedef struct smaug_params {
  int32_t version;          /* SMAUG_PARAMS_VERSION */
  int32_t ndim;             /* 2 or 3 */
  int32_t n[3];             /* p->n: cells per dim including ghosts (n[2]=1 in 2D) */
  int32_t moddton;          /* p->moddton: 1 = adaptive dt from the CFL max */
  int32_t hyperdifmom;      /* p->hyperdifmom: 1 = hyperdiffusion on */
  int32_t integrator;       /* SMAUG_INT_* */
  int32_t precision;        /* SMAUG_PREC_* */
  int32_t pad_model;        /* SMAUG_PAD_* */
  int32_t boundtype[3][2];  /* p->boundtype[*][dim][0]=upper, [1]=lower */
  int32_t driver;           /* SMAUG_DRIVER_* */
  int32_t stencil_order;    /* flux-divergence derivative grad3dn: 4 (or 0) the
                               4th-order default, 6 the reference's USE_DORDER3
                               build (src/gradops.cu:450-453) */
  int32_t drv_step;         /* SMAUG_DRIVER_GAUSS_STEP: the step counter value at
                               which the driver acts */
  int32_t reserved_i[5];
  double dx[3];             /* p->dx: (xmax-xmin)/(n-4), used by the dt rule */
  double dt;                /* p->dt at start (the reference sets 1e-8 when moddton) */
  double dtmax;             /* DT: adaptive dt is accepted only below this */
  double courant;           /* p->courant */
  double gamma;             /* p->gamma */
  double eta;               /* p->eta (written to .out headers only) */
  double g[3];              /* p->g: gravity */
  double chyp[SMAUG_MAXVAR];/* p->chyp[field]: hyperdiffusion coefficients */
  double xmin[3];           /* p->xmin (used by the .out writer metadata only) */
  /* Gaussian driver: v = amp * sin(2 pi t / period) * prod_d exp(-((x_d-x0_d)/sigma_d)^2)
     over dims with sigma_d > 0; period <= 0 means a steady driver. */
  double drv_amp, drv_period;
  double drv_x0[3];
  double drv_sigma[3];
  double reserved_d[8];
} smaug_params_t;

typedef struct smaug_engine* smaug_handle_t;

/* Fill *p with the reference's Orszag-Tang defaults for an N0 x N1 interior
   (models/iosmaugparams.h.ot): gamma 5/3, chyp 0.2, periodic, moddton. */
int smaug_params_default(smaug_params_t* p, int32_t ndim);

/*
 * Create an engine on the current CUDA device.  Replaces cuinit
 * (src/init.cu:2222-2448) + initgrid (src/init.cu:2502-3060) + the initial
 * cuboundary sweep (src/iosmaug.c:480-488).
 *   w   : NVAR*ncells doubles, reference layout (slot 0 as read from .ini)
 *   pos : NDIM*ncells doubles, cell positions (wd[pos1..] of the reference)
 */
int smaug_create(const smaug_params_t* p, const double* w, const double* pos,
                 smaug_handle_t* out);

/* Advance nsteps steps.  Replaces the body of the step loop
   src/iosmaug.c:496-1144 (cucomputedervfields ... cuboundary). */
int smaug_step(smaug_handle_t h, int32_t nsteps);

/* Enqueue nsteps steps on the engine's stream without waiting; the
   non-finite check is reported by the next smaug_sync.  For capture in CUDA
   graphs and for timing with events on the caller's stream. */
int smaug_step_async(smaug_handle_t h, int32_t nsteps);

/* Wait for the engine's stream; returns SMAUG_E_NONFINITE if a NaN/Inf was
   produced since the last check. */
int smaug_sync(smaug_handle_t h);

/* Launch on `stream` (a cudaStream_t) from now on; NULL restores the
   engine's own stream.  The caller keeps ownership of the stream. */
int smaug_set_stream(smaug_handle_t h, void* stream);

/* Copy the current state (all NVAR fields, ghosts included) to the host.
   Replaces cuupdate (src/update.cu:165-233). */
int smaug_get_state(smaug_handle_t h, double* w);

/* Copy fields [f0, f0+nf) of the current state (reference numbering) to the
   host, field-major, w pointing at the destination of field f0 -- e.g. only
   the evolved fields after a step.  A subset of smaug_get_state (cuupdate
   copies every field of two slots, src/update.cu:207). */
int smaug_get_fields(smaug_handle_t h, double* w, int32_t f0, int32_t nf);

/* Replace the evolved fields from a host array in reference layout. */
int smaug_set_state(smaug_handle_t h, const double* w);

/* Step counter, simulated time and the dt of the last step (state->it, t, dt). */
int smaug_get_time(smaug_handle_t h, int64_t* it, double* t, double* dt);

/* Per-dimension CFL maxima of the current state (p->cmax per dim,
   src/computedervfields.cu:1864-2050). */
int smaug_get_cmax(smaug_handle_t h, double* cmax);

/* How the 2D stage kernel stages its tiles in shared memory: *tma = 0
   per-thread loads, 1 bulk tensor copies (TMA) in a persistent grid whose
   blocks copy their next tile during the current one's stores, 2 bulk
   tensor copies with one block per tile; *available = 1 when the grid
   admits the copies (2D, rows a multiple of 16 bytes in the storage type,
   4th-order stencil).  Either pointer may be null.  No reference
   counterpart: the reference stages no tiles. */
int smaug_staging(smaug_handle_t h, int32_t* tma, int32_t* available);
/* Select the staging of subsequent launches (0, 1 or 2 as above); the
   results are bitwise identical.  SMAUG_E_UNSUPPORTED when 1 or 2 is asked
   for and not available. */
int smaug_set_staging(smaug_handle_t h, int32_t tma);

/* Write the current state as a reference .out file (src/readwrite.c:160-366).
   `it` and `t` go to the header; name is the 79-byte run name. */
int smaug_write_out(smaug_handle_t h, const char* path, const char* name,
                    int32_t it, double t);

/* Asynchronous snapshot (the reference writes .out files synchronously from
   the step loop, src/iosmaug.c:509-517 writevacconfig): enqueue the copy of
   the current state on the engine's stream into a pinned host buffer and
   return; a host thread writes the .out file when the copy has completed,
   while the caller keeps stepping.  Two buffers are used in turn, so a third
   call first waits for the oldest write.  Errors of the write itself are
   reported by smaug_wait_writes. */
int smaug_write_out_async(smaug_handle_t h, const char* path, const char* name,
                          int32_t it, double t);

/* Wait for every pending asynchronous write; returns the first write error
   since the last call (SMAUG_E_IO with the file's message), else 0.
   smaug_destroy waits as well. */
int smaug_wait_writes(smaug_handle_t h);

/* Release all device memory of the handle. */
int smaug_destroy(smaug_handle_t h);

/* ---- batched ensemble of independent 2D runs ----------------------------
 * No counterpart in the reference (one run per process there).  Runs of any
 * size, boundary types, background fields and driver advance together with
 * classical RK4 over the tile list of all runs, in one of two forms: one
 * launch per stage, or one persistent launch for several steps whose blocks
 * take tiles from a shared counter and meet at a grid barrier between stages.
 * A cycle of 6 steps is captured once into a CUDA graph and replayed (24 stage
 * launches, or one persistent launch).  All runs share one precision form.
 * The first 10 steps time 2 tile shapes (32x8, 16x16) x 5 launch shapes (1 and
 * 2 blocks per SM, the occupancy limit per SM, one block per tile, the
 * persistent launch) and keep the fastest; results do not depend on either
 * shape.  Each run's results equal those of the same run stepped alone with
 * smaug_step. */
typedef struct smaug_batch_s* smaug_batch_t;

/* params[r], w[r], pos[r]: as smaug_create for run r (2D, integrator RK4) */
int smaug_batch_create(int32_t nruns, const smaug_params_t* const* params, const double* const* w,
                       const double* const* pos, smaug_batch_t* out);
/* advance every run by nsteps RK4 steps; waits and reports non-finite values */
int smaug_batch_step(smaug_batch_t b, int32_t nsteps);
/* enqueue without waiting / wait and report; launch on a caller stream (NULL:
   the batch's own) */
int smaug_batch_step_async(smaug_batch_t b, int32_t nsteps);
int smaug_batch_sync(smaug_batch_t b);
int smaug_batch_set_stream(smaug_batch_t b, void* stream);
/* state / time of run `run`, as smaug_get_state / smaug_get_time */
int smaug_batch_get_state(smaug_batch_t b, int32_t run, double* w);
int smaug_batch_get_time(smaug_batch_t b, int32_t run, int64_t* it, double* t, double* dt);
/* chosen grid (0 before tuning), the 4 candidate grids of the chosen tile
   shape and their step times in ms */
int smaug_batch_launch_shape(smaug_batch_t b, int32_t* grid, int32_t* candidates, float* ms);
/* The batch's first steps time every (tile shape, grid) candidate and keep the
   fastest: tile shapes 32x8 and 16x16, 4 grids each.  Chosen tile (0x0 before
   tuning) and the 8 step times in ms (32x8's four grids, then 16x16's; 0 for
   a candidate not timed). */
int smaug_batch_tile_shape(smaug_batch_t b, int32_t* tx, int32_t* ty, float* ms);
/* Use only tile shape tx x ty (32x8 or 16x16); call before the first step. */
int smaug_batch_pin_tile_shape(smaug_batch_t b, int32_t tx, int32_t ty);
/* The persistent launch: *on = 1 when the tuner chose it; grid[2] its blocks
   and ms[2] its step time per tile shape (32x8, 16x16; 0 when not timed). */
int smaug_batch_persistent(smaug_batch_t b, int32_t* on, int32_t* grid, float* ms);
/* Restrict the tuner to one form: -1 both (default), 0 per-stage launches,
   1 the persistent launch; call before the first step. */
int smaug_batch_pin_form(smaug_batch_t b, int32_t form);
int smaug_batch_destroy(smaug_batch_t b);

/* ---- adjoint of one RK4 step (2D, FP64, dt held fixed) -------------------
 * No counterpart in the reference (which has no derivatives).  The step is
 * u -> U' = RK4 step of G(u) (G: ghost fill) with dt = p->dt fixed
 * (p->moddton must be 0), the hyperdiffusion coefficient's maxima and the CFL
 * maxima differentiated through the cells that attain them.  States are
 * DEVICE arrays of the 2D evolved fields [6][n1*n0] in reference layout; the
 * background fields are taken from w at create.  Driver parameters theta =
 * (amplitude, period, centre along dim 1). */
typedef struct smaug_adj_s* smaug_adj_t;

int smaug_adj_create(const smaug_params_t* p, const double* w, const double* pos, smaug_adj_t* out);
/* theta of the driver term (overrides p's drv_amp, drv_period, drv_x0[1]) */
int smaug_adj_set_driver(smaug_adj_t a, double amp, double period, double x0);
/* u_next = step(u) at time t; enqueued on `stream` */
int smaug_adj_forward(smaug_adj_t a, const double* u, double* u_next, double t, void* stream);
/* ubar = (dU'/du)^T ubar_next, thbar[3] = (dU'/dtheta)^T ubar_next (device
   arrays, overwritten); recomputes the step's stages; enqueued on `stream` */
int smaug_adj_backward(smaug_adj_t a, const double* u, const double* ubar_next, double* ubar,
                       double* thbar, double t, void* stream);
/* Tape of nslots steps (4 x 6 x ncells doubles each): a taped forward keeps
   the step's stage inputs, so the matching backward recomputes nothing.
   Grows only (waits for the device when it reallocates). */
int smaug_adj_tape_reserve(smaug_adj_t a, int32_t nslots);
/* smaug_adj_forward, keeping the stage inputs in tape slot `slot` */
int smaug_adj_forward_tape(smaug_adj_t a, const double* u, double* u_next, double t, int32_t slot,
                           void* stream);
/* smaug_adj_backward of the step taped in `slot` (same t) */
int smaug_adj_backward_tape(smaug_adj_t a, int32_t slot, const double* ubar_next, double* ubar,
                            double* thbar, double t, void* stream);

/* The step adjoints of taped slots slot_lo .. slot_lo+nsteps-1 in reverse
   order in one call, for the steps n_lo .. n_lo+nsteps-1 of a rollout (step
   n at time t0 + n*dt).  ubar: in, the adjoint of the state after the last
   step; out, the adjoint of the state before the first.  Before the adjoint
   of step n_lo+k, gsteps[k] (6*ncell doubles, e.g. the gradient of a loss
   term at that step's output) is added to it, when gsteps is not NULL.
   thbar (3 doubles) accumulates the parameter adjoints (not cleared). */
int smaug_adj_backward_tape_range(smaug_adj_t a, int32_t slot_lo, int32_t nsteps,
                                  const double* gsteps, double* ubar, double* thbar,
                                  double t0, int32_t n_lo, void* stream);
int smaug_adj_destroy(smaug_adj_t a);

/* Message of the calling thread's last failure ("" if none). */
const char* smaug_last_error(void);

/* Library version string. */
const char* smaug_version(void);

/*
 * One reference (Euler) step that allocates nothing.  No counterpart in the
 * reference.  It is for callers that cannot call cudaMalloc: applications
 * that reserve their device memory up front (a caching pool, a fixed budget
 * on a shared GPU) and cannot satisfy or do not allow allocations made behind
 * their back, plugins whose host forbids allocation inside its step callback,
 * and loops running beside other streams that cudaFree's implicit device-wide
 * synchronisation would stall.
 *   w_in, w_out : DEVICE buffers, NVAR*ncells doubles each, reference layout;
 *                 w_in needs valid ghost layers (as left by a previous step);
 *                 w_out receives the whole state (backgrounds copied).
 *   delx        : HOST array of n[0]+n[1] doubles, the cell widths along dim 0
 *                 then dim 1 (one interior line of smaug_grid_metric's output).
 *   dt          : HOST in/out: the previous step's dt in, this step's dt out.
 *   stream      : cudaStream_t or NULL.
 * 2D only, no driver term, at most 8192 cells per dimension (ghosts
 * included); larger grids are rejected with SMAUG_E_UNSUPPORTED.  Scratch
 * lives in one static device array of 196,864 bytes per GPU, kept until the
 * process exits and shared by every call, which clears the parts that must
 * start at zero: calls whose GPU work overlaps (other threads or streams)
 * race on it and must be serialised by the caller.  The first call on a
 * device looks up that array's device address and keeps it for the rest of
 * the process (so it does not survive a cudaDeviceReset); make that first
 * call before any stream capture.  Returns after the step completed.
 */
int smaug_euler_step_noalloc(const smaug_params_t* p, const double* w_in, double* w_out,
                             const double* delx, double* dt, void* stream);

/*
 * Format boundary (host only, no device use).
 * Read a reference ASCII .ini (src/readwrite.c:975-1082): header + one line
 * per cell "pos[ndim] w[nvar]".  n[] must be set by the caller (the reference
 * takes it from compile-time NI/NJ); the file's own n line is checked.
 */
int smaug_read_ini(const char* path, int32_t ndim, const int32_t* n,
                   double* w, double* pos, int32_t* it, double* t);

/* Write a reference binary .out (src/readwrite.c:160-366) from host arrays. */
int smaug_write_out_host(const char* path, const smaug_params_t* p,
                         const double* w, const double* pos, const char* name,
                         int32_t it, double t);

/* Grid metric from positions (host), the reference's initgrid
   (src/init.cu:2502-3060): rewrites ghost positions by linear extrapolation
   and fills delx[d*ncells + cell]. */
int smaug_grid_metric(int32_t ndim, const int32_t* n, double* pos, double* delx);

#ifdef __cplusplus
}
#endif

#endif /* SMAUG_B200_H_ */
