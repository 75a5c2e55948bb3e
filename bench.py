"""Benchmark of the SMAUG time advance on B200 (one JSON line on rank 0).

Workload (N=1): 2D Orszag-Tang vortex, 4096 x 4096 interior cells (+2 ghost
layers), periodic, hyperdiffusion on, CFL 0.3, seeded 1e-3 rho noise, FP64,
classical RK4 -- the bandwidth/roofline configuration of the benchmark suite.
A step is one RK4 step (4 fused stage launches).  The state (0.8 GB per
buffer) is far larger than the 126 MB L2, so no flush is needed between steps.

  value  Mcell-updates/s per RK4 step, state resident in HBM, CUDA events on
         the engine's stream (torch's current stream is handed to the engine)
  e2e    the same metric through the C ABI with host buffers: per step
         smaug_set_state (pinned H2D of the evolved fields) + smaug_step +
         smaug_get_fields (D2H of the evolved fields)
  mixed  the mixed precision form (float perturbation storage and
         hyperdiffusion, double elsewhere) on the same workload, timed the
         same way, with its relative L2 distance per field from the FP64
         state after the same number of steps
N>1 (torchrun): replicas only -- each rank advances its own copy, no
collective on the data path; value = total cell updates / max rank time.

--workload tube: the 3D stratified solar atmosphere instead (256^3 interior
cells by default, --n sets it): vertical axis = dim 0 (contcd4 ghosts),
periodic x and y, hydrostatic background on 2 x 2 x 6 Mm with a uniform
10 G vertical field, Gaussian vertical-velocity driver (200 m/s, 30 s period,
sigma 0.2 Mm, centred at z = 0.1 Mm, x = y = 1 Mm), gravity 274 m/s^2.

--workload ensemble: 64 uneven 2D runs (sizes drawn by seed from 64^2..512^2,
Orszag-Tang and stratified driven slabs) advanced by one batch (one launch per
stage for all runs, CUDA-graph cycles, autotuned launch shape), against the
same runs stepped one by one; mixed precision unless --precision fp64.

--workload adjoint: the driver-parameter gradient of a 400-step loss on a
256 x 512 stratified slab through the hand-written adjoint (checkpoints every
20 steps): adjoint-to-forward cost ratio and the finite-difference check.

--impl reference: the reference has no CPU solver (every routine is a CUDA
kernel), so the CPU baseline is the oracle, the FP64 restatement of the
reference's kernels (oracle/), run with all host threads on a bounded
sample of the same workload.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD_N = 4096
TUBE_N = 256
METRIC = "Mcell-updates/s per RK4 step"
UNIT = "Mcell-updates/s"


# DRAM bytes per interior cell per RK4 step measured by ncu on the four stage
# launches of one step at the benchmark sizes (profiles/dram_traffic_per_stage.md:
# 2D at 4096^2, 3D at 256^3)
TRAFFIC_PER_CELL_STEP = {(2, "fp64"): 889.1, (2, "mixed"): 745.7, (3, "fp64"): 2241.6,
                         (3, "mixed"): 1510.6}

# What bounds each stage kernel, from its ncu section set (profiles/)
BOUND_NOTE = {
    (2, "fp64"): "issue-bound, not HBM: 109 warp instructions per cell and stage at 59.8 % issue "
                 "active, FP64 pipe 35 %, barrier stalls 2.9 per issue "
                 "(profiles/stage2d_fp64_ot2048_full.md)",
    (2, "mixed"): "issue-bound, not HBM: 102 warp instructions per cell and stage at 60.5 % issue "
                  "active (profiles/stage2d_mixed_ot2048_full.md)",
    (3, "fp64"): "latency/issue-bound, not HBM: 494 warp instructions per cell and stage at 47.8 % "
                 "issue active, long-scoreboard stalls 3.65 per issue from re-reads of the state, "
                 "DRAM traffic 1.8x the algorithmic bytes (profiles/stage3d_fp64_tube128_full.md)",
    (3, "mixed"): "latency/issue-bound, not HBM: as the FP64 form, with float storage "
                  "(profiles/stage3d_fp64_tube128_full.md)",
}

# FP64 (and FP32) floating-point operations per interior cell per stage counted
# by ncu (smsp__sass_thread_inst_executed_op_{dadd,dmul,dfma}_pred_on, an FMA
# counting 2; profiles/fp64_flops_per_cell.md: 2D at 2048^2, 3D at 128^3)
FLOP_PER_CELL_STAGE = {(2, "fp64"): (1208.0, 29.0), (2, "mixed"): (566.0, 424.0),
                       (3, "fp64"): (3731.0, 107.0)}


def fp64_roofline(ndim, prec, ncell, steps, ms):
    """Secondary roofline of a stage kernel against the nominal FP64 vector
    peak (148 SMs x 64 FP64 FMA per clock x 2 at the maximum SM clock)."""
    fl = FLOP_PER_CELL_STAGE.get((ndim, prec))
    if fl is None:
        return None
    mhz = 1965.0
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        mhz = float(json.load(open(path)).get("sm_max_mhz", mhz))
    peak = 148 * 64 * 2 * mhz * 1e6 / 1e12
    ach = fl[0] * 4 * ncell * steps / (ms / 1e3) / 1e12
    return {"bound": "fp64", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
            "fp64_flop_per_cell_stage": fl[0], "fp32_flop_per_cell_stage": fl[1],
            "peak_kind": "nominal: 148 SMs x 64 FP64 FMA/clk x 2 x %.0f MHz" % mhz}


def alg_bytes_per_cell_step(ndim):
    """Algorithmic HBM bytes per interior cell per RK4 step, FP64, by the
    benchmark's accounting for a minimal three-register classical RK4 with
    every stage fused: stage 1 reads Un,B and writes U2,Acc; stages 2-3 read
    Us,Un,Acc,B and write Us+1,Acc; stage 4 reads U4,Un,Acc,B and writes Un+1
    -> 17P+4B doubles for P evolved and B background fields (2D: 944, 3D:
    1248)."""
    P, B = 2 + 2 * ndim, 2 + ndim
    return (17 * P + 4 * B) * 8


def alg_bytes_mixed(ndim):
    """The same accounting with the mixed form's element sizes: stage states
    in float (4 B), the base state Un and Un+1 as a float high/low pair (8 B),
    accumulator and backgrounds in double -> 112P+32B bytes (2D: 800, 3D:
    1056)."""
    P, B = 2 + 2 * ndim, 2 + ndim
    return 112 * P + 32 * B


def scheme_bytes_per_cell_step(ndim, mixed=False):
    """Bytes this engine's scheme moves: its accumulator starts as
    Un + k1/6, so stage 4 does not read Un again -> 16P+4B doubles (2D: 896,
    3D: 1184); mixed 100P+32B (2D: 728, 3D: 960)."""
    P, B = 2 + 2 * ndim, 2 + ndim
    return 100 * P + 32 * B if mixed else (16 * P + 4 * B) * 8


def roofline_block(ndim, prec, alg_bytes, ncell, steps, ms, peak, peak_kind):
    """HBM roofline of the stage kernel: achieved = algorithmic bytes per
    interior cell and step x cells x steps / device time; traffic = the DRAM
    bytes ncu measured per stage launch at this size, and the bandwidth the
    kernel actually drew from them (achieved_by_traffic)."""
    achieved = alg_bytes * ncell * steps / (ms / 1e3) / 1e9
    tcell = TRAFFIC_PER_CELL_STEP.get((ndim, prec))
    out = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
           "peak_kind": peak_kind, "alg_bytes_per_cell_step": alg_bytes,
           "scheme_bytes_per_cell_step": scheme_bytes_per_cell_step(ndim, prec == "mixed"),
           "traffic": tcell * ncell / 4 if tcell else None,
           "traffic_unit": "DRAM bytes per stage launch (ncu at the benchmark size)",
           "note": BOUND_NOTE.get((ndim, prec))}
    if tcell:
        by_traffic = tcell * ncell * steps / (ms / 1e3) / 1e9
        out["achieved_by_traffic"] = by_traffic
        out["frac_by_traffic"] = by_traffic / peak
    return out


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks/throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0, period_ms=50):
        self.index = index
        self.period_ms = period_ms
        self.samples = []
        self._p = None

    def __enter__(self):
        # one nvidia-smi in loop mode (-lms), the process this object started
        try:
            self._p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            # the first sample arrives once nvidia-smi is up: the timed
            # region starts after it, and it is not counted
            self._p.stdout.readline()
        except Exception:
            self._p = None
        return self

    def __exit__(self, *a):
        if self._p is None:
            return
        self._p.terminate()
        try:
            out, _ = self._p.communicate(timeout=10)
        except Exception:
            self._p.kill()
            out, _ = self._p.communicate()
        for ln in (out or "").strip().splitlines():
            f = [x.strip() for x in ln.split(",")]
            if len(f) >= 5:
                self.samples.append(f)

    def summary(self):
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def make_case(N, seed=1, precision=0):
    from smaug_b200 import ic, params as P
    w, pos, dx = ic.orszag_tang(N, noise=1e-3, seed=seed)
    p = P.make_params(ndim=2, n=(N + 4, N + 4, 1), dx=dx, courant=0.3, dtmax=1.0,
                      integrator=P.INT_RK4, precision=precision)
    return p, w, pos


def make_tube(N, seed=1, precision=0):
    """3D stratified atmosphere, N^3 interior cells, 2 x 2 x 6 Mm (dim 0 vertical)."""
    from smaug_b200 import ic, params as P
    w, pos, dx = ic.stratified(nz=N, nx=N, ny=N, seed=seed)
    p = P.make_params(ndim=3, n=(N + 4, N + 4, N + 4), dx=dx, courant=0.3, dtmax=1.0,
                      integrator=P.INT_RK4, g=(-274.0, 0.0, 0.0), precision=precision,
                      boundtype=(P.BC_CONTCD4, P.BC_PERIODIC, P.BC_PERIODIC),
                      driver=P.DRIVER_GAUSS, drv_amp=200.0, drv_period=30.0,
                      drv_x0=(0.1e6, 1.0e6, 1.0e6), drv_sigma=(0.2e6, 0.2e6, 0.2e6))
    return p, w, pos


def workload(args, seed=1):
    """(params, w, pos, interior cells, description) of the selected workload."""
    N = args.n
    prec = 1 if args.precision == "mixed" else 0
    if args.workload == "tube":
        p, w, pos = make_tube(N, seed, prec)
        p.stencil_order = args.stencil_order
        return p, w, pos, N ** 3, ("3D stratified atmosphere %dx%dx%d (+2 ghost layers), 2x2x6 Mm, "
                                   "contcd4 vertical / periodic horizontal, gravity, Gaussian "
                                   "driver, hyperdiffusion, CFL 0.3, FP64, classical RK4" % (N, N, N))
    p, w, pos = make_case(N, seed, prec)
    p.stencil_order = args.stencil_order
    return p, w, pos, N * N, ("2D Orszag-Tang %dx%d (+2 ghost layers), periodic, "
                              "hyperdiffusion, CFL 0.3, FP64, classical RK4" % (N, N))


ENSEMBLE_SIZES = (64, 128, 192, 256, 384, 512)


def make_ensemble(nruns=64, seed=5, precision=1):
    """Uneven 2D runs: sizes drawn by seed from ENSEMBLE_SIZES, alternately
    Orszag-Tang (seeded rho noise) and stratified driven slabs (2 x 6 Mm,
    vertical dim 0, driver periods uniform in [10, 300] s), RK4."""
    import numpy as np
    from smaug_b200 import ic, params as P
    rng = np.random.default_rng(seed)
    runs = []
    for r in range(nruns):
        n = int(rng.choice(ENSEMBLE_SIZES))
        if r % 2 == 0:
            w, pos, dx = ic.orszag_tang(n, noise=1e-3, seed=seed + r)
            p = P.make_params(ndim=2, n=(n + 4, n + 4, 1), dx=dx, courant=0.3, dtmax=1.0,
                              integrator=P.INT_RK4, precision=precision)
        else:
            period = float(rng.uniform(10.0, 300.0))
            w, pos, dx = ic.stratified(nz=n, nx=n, seed=seed + r, vz_sigma=10.0)
            p = P.make_params(ndim=2, n=(n + 4, n + 4, 1), dx=dx, courant=0.3, dtmax=1.0,
                              integrator=P.INT_RK4, precision=precision, g=(-274.0, 0.0),
                              boundtype=(P.BC_CONTCD4, P.BC_PERIODIC), driver=P.DRIVER_GAUSS,
                              drv_amp=200.0, drv_period=period, drv_x0=(0.1e6, 1.0e6),
                              drv_sigma=(0.2e6, 0.2e6))
        runs.append((p, w, pos, n * n))
    return runs


def ensemble_main(args):
    """--workload ensemble: 64 uneven runs in one batch (per-stage or persistent
    launches for all runs, 6-step CUDA graph cycles, autotuned tile shape and
    launch form) against the same runs stepped one by one through their own
    engines; each launch form is also timed alone (`forms`)."""
    import torch
    from smaug_b200 import engine
    prec = 0 if args.precision == "fp64" else 1
    runs = make_ensemble(args.nruns, precision=prec)
    cells = sum(r[3] for r in runs)
    # the first 10 steps time the (tile shape, launch) candidates; the 6-step
    # CUDA graph is captured at the next cycle boundary with a full cycle to
    # go, so 24 warm-up steps leave capture and instantiation out of the
    # timed steps
    warm = max(args.warmup, 24)
    stream = torch.cuda.Stream()

    def timed_batch(form):
        b = engine.Batch([r[0] for r in runs], [r[1] for r in runs], [r[2] for r in runs])
        b.set_stream(stream.cuda_stream)
        b.pin_form(form)
        b.step(warm)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(0) as clk:
            ev0.record(stream)
            b.step_async(args.steps)
            ev1.record(stream)
            torch.cuda.synchronize()
        b.sync()
        shape = b.launch_shape()
        shape["tile"] = b.tile_shape()
        shape["persistent"] = b.persistent()
        b.close()
        return ev0.elapsed_time(ev1), shape, clk

    ms, shape, clk = timed_batch(None)           # the autotuner's choice
    forms = {}
    for form in ("per-stage", "persistent"):     # each form alone, steady state
        fms, fshape, _ = timed_batch(form)
        forms[form] = {"value": cells * args.steps / (fms / 1e3) / 1e6, "unit": UNIT,
                       "ms_per_step": fms / args.steps, "tile": fshape["tile"]["tile"],
                       "grid": fshape["grid"]}
    # one by one: each run alone, its own engine and stream, same step counts
    ms_single = 0.0
    for p, w, pos, nc in runs:
        e = engine.Engine(p, w, pos)
        e.set_stream(stream.cuda_stream)
        e.step(warm)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        e.step_async(args.steps)
        ev1.record(stream)
        e.sync()
        torch.cuda.synchronize()
        ms_single += ev0.elapsed_time(ev1)
        e.close()
    value = cells * args.steps / (ms / 1e3) / 1e6
    single = cells * args.steps / (ms_single / 1e3) / 1e6
    peak, pk_kind = peaks()
    mbytes = alg_bytes_mixed(2) if prec else alg_bytes_per_cell_step(2)
    achieved = mbytes * cells * args.steps / (ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": warm, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 storage + hyperdiffusion, f64 rest" if prec else "f64",
        "data": "synthetic",
        "config": {"workload": "ensemble of %d uneven 2D runs (sizes from %s by seed, "
                               "Orszag-Tang and stratified driven slabs), classical RK4"
                               % (len(runs), list(ENSEMBLE_SIZES)),
                   "interior_cells": cells, "sizes": [int(round(r[3] ** 0.5)) for r in runs],
                   "precision": args.precision,
                   "timing": "CUDA events on the launch stream, batch and each single run"},
        "one_by_one": {"value": single, "unit": UNIT, "ms_per_step": ms_single / args.steps},
        "speedup_vs_one_by_one": value / single,
        "launch_shape": shape,
        "forms": forms,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "alg_bytes_per_cell_step": mbytes,
                     "scheme_bytes_per_cell_step": scheme_bytes_per_cell_step(2, bool(prec)),
                     "peak_kind": pk_kind},
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def make_slab(nx=256, nz=512, seed=11):
    """2D stratified slab 256 (x) x 512 (z), 2 x 6 Mm, vertical dim 0, seeded
    FP32 v_z perturbation (sigma 10 m/s, Gaussian-smoothed over 3 cells),
    Gaussian driver (200 m/s, 30 s, x0 = 1 Mm, z = 0.1 Mm, sigma 0.2 Mm)."""
    from smaug_b200 import ic, params as P
    w, pos, dx = ic.stratified(nz=nz, nx=nx, seed=seed, vz_sigma=10.0)
    p = P.make_params(ndim=2, n=(nz + 4, nx + 4, 1), dx=dx, courant=0.3, dtmax=1.0,
                      integrator=P.INT_RK4, g=(-274.0, 0.0),
                      boundtype=(P.BC_CONTCD4, P.BC_PERIODIC), driver=P.DRIVER_GAUSS,
                      drv_amp=200.0, drv_period=30.0, drv_x0=(0.1e6, 1.0e6),
                      drv_sigma=(0.2e6, 0.2e6))
    return p, w, pos


def adjoint_main(args):
    """--workload adjoint: gradient of sum_n sum_x (v_z(z = 3 Mm) - target)^2
    over 400 RK4 steps with respect to the driver (amplitude, period, x0),
    through the hand-written adjoint with checkpoints every 20 steps; the
    target comes from a forward run with seed-shifted parameters.  Reports the
    forward and forward+backward times (CUDA events), their ratio, and the
    central finite-difference check (h = 1e-4 relative) of every component,
    for the taped rollout and (composed_checkpoint_autograd) for single-step
    Functions under torch.utils.checkpoint.  No driver signal reaches the
    3 Mm row within 400 steps of half the CFL dt (the loss there is exactly
    0), so the same measurement is repeated for the row at 0.4 Mm."""
    import numpy as np
    import torch
    from smaug_b200 import engine, params as P
    from smaug_b200.adjoint import StepAdjoint, rollout, rollout_autograd
    nsteps = args.adj_steps
    p, w, pos = make_slab()
    e = engine.Engine(p, w, pos)
    e.step(1)
    dt = e.time()[2]
    e.close()
    q = P.SmaugParams.from_buffer_copy(p)
    q.moddton = 0
    q.dt = 0.5 * dt
    sa = StepAdjoint(q, w, pos)
    u0 = torch.tensor(w[:6], dtype=torch.float64, device="cuda").contiguous()
    rhob = torch.tensor(w[7], device="cuda", dtype=torch.float64)
    theta0 = torch.tensor([200.0, 30.0, 1.0e6], dtype=torch.float64)
    rng = np.random.default_rng(12)
    shift = torch.tensor(1.0 + 0.05 * rng.standard_normal(3), dtype=torch.float64)
    line = None
    # the headline row is 0.4 Mm; the configured 3 Mm row is reported beside it
    # and labelled: nothing the driver excites reaches it within 400 steps
    for obs_z in [args.obs_z] + ([3.0e6] if abs(args.obs_z - 3.0e6) > 1.0 else []):
        res = _adjoint_case(args, sa, q, p, u0, pos, rhob, theta0, shift, obs_z, nsteps,
                            rollout, rollout_autograd)
        if line is None:
            line = res
        else:
            sub = {k: res[k] for k in ("value", "loss", "grad", "forward_ms", "forward_backward_ms")}
            sub["observed_row_z_m"] = res["config"]["observed_row_z_m"]
            if res["loss"] == 0.0:
                sub["degenerate"] = ("no signal reaches the row within the rollout: loss and gradient "
                                     "are exactly 0 and every adjoint tile returns at its first barrier")
            line["configured_row_3Mm"] = sub
    sa.close()
    print(json.dumps(line), flush=True)


def _adjoint_case(args, sa, q, p, u0, pos, rhob, theta0, shift, obs_z, nsteps, rollout,
                  rollout_autograd):
    import numpy as np
    import torch
    kz = int(np.argmin(np.abs(pos[0][0] - obs_z)))

    def vz_row(u):
        return u[1, :, kz] / (u[0, :, kz] + rhob[:, kz])

    with torch.no_grad():
        sa.set_driver(*(theta0 * shift).tolist())
        target, u = [], u0
        for n in range(nsteps):
            u = sa.forward(u, n * q.dt)
            target.append(vz_row(u).clone())

    def loss_fn(u, n):
        return ((vz_row(u) - target[n - 1]) ** 2).sum()

    def timed(fn):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        out = fn()
        b.record()
        torch.cuda.synchronize()
        return out, a.elapsed_time(b)

    for _ in range(max(args.warmup, 1)):
        with torch.no_grad():
            rollout(sa, theta0, u0, 20, loss_fn, checkpoint_every=20)
    # one full backward of each rollout outside the timed regions (the tape
    # is allocated on the first backward, and torch's caching allocator
    # grows to the rollout's working set)
    for fn, every in ((rollout, 20), (rollout_autograd, 20), (rollout, 0)):
        thw = theta0.clone().requires_grad_(True)
        fn(sa, thw, u0, nsteps, loss_fn, checkpoint_every=every).backward()
    with torch.no_grad():
        L0, ms_fwd = timed(lambda: rollout(sa, theta0, u0, nsteps, loss_fn, checkpoint_every=20))

    def fwd_bwd():
        th = theta0.clone().requires_grad_(True)
        L = rollout(sa, th, u0, nsteps, loss_fn, checkpoint_every=20)
        L.backward()
        return th.grad.clone()

    grad, ms_fb = timed(fwd_bwd)

    def fwd_bwd_composed():
        th = theta0.clone().requires_grad_(True)
        L = rollout_autograd(sa, th, u0, nsteps, loss_fn, checkpoint_every=20)
        L.backward()
        return th.grad.clone()

    grad_c, ms_fb_c = timed(fwd_bwd_composed)

    def fwd_bwd_full_tape():
        th = theta0.clone().requires_grad_(True)
        L = rollout(sa, th, u0, nsteps, loss_fn, checkpoint_every=0)
        L.backward()
        return th.grad.clone()

    grad_t, ms_fb_t = timed(fwd_bwd_full_tape)
    def central_fd(hrel):
        out = []
        for k in range(3):
            h = hrel * float(theta0[k])
            vals = []
            for sgn in (1, -1):
                th = theta0.clone()
                th[k] += sgn * h
                with torch.no_grad():
                    vals.append(float(rollout(sa, th, u0, nsteps, loss_fn, checkpoint_every=20)))
            out.append((vals[0] - vals[1]) / (2 * h))
        return out

    def rel_err(fd):
        return [abs(float(grad[k]) - fd[k]) / max(abs(fd[k]), 1e-300) for k in range(3)]

    fd = central_fd(1e-4)          # the configured step
    rel = rel_err(fd)
    fd6 = central_fd(1e-6)         # closer to the limit (truncation error ~h^2)
    rel6 = rel_err(fd6)
    cells = p.interior_cells()
    line = {
        "metric": "adjoint cost / forward cost (loss gradient over a 400-step RK4 rollout)",
        "value": ms_fb / ms_fwd, "unit": "x forward", "n_gpus": 1, "steps": nsteps, "warmup": args.warmup,
        "ms_per_step": ms_fb / nsteps, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "2D stratified slab 256x512, driver gradient, dt fixed, "
                               "checkpoints every 20 steps", "interior_cells": cells,
                   "observed_row_z_m": float(pos[0][0][kz]), "dt_s": q.dt},
        "forward_ms": ms_fwd, "forward_backward_ms": ms_fb,
        "forward_mcell_updates_per_s": cells * nsteps / (ms_fwd / 1e3) / 1e6,
        "loss": float(L0), "grad": [float(g) for g in grad], "fd": fd, "fd_rel_err": rel,
        "fd_h": 1e-4, "fd_h1e-6": {"fd": fd6, "fd_rel_err": rel6},
        "composed_checkpoint_autograd": {
            "value": ms_fb_c / ms_fwd, "forward_backward_ms": ms_fb_c,
            "grad": [float(g) for g in grad_c],
            "note": "single-step Functions under torch.utils.checkpoint; each step adjoint "
                    "recomputes its stage inputs"},
        "full_tape": {
            "value": ms_fb_t / ms_fwd, "forward_backward_ms": ms_fb_t,
            "grad": [float(g) for g in grad_t],
            "grad_max_rel_diff_vs_checkpointed": float((grad_t - grad).abs().max() / grad.abs().max())
            if float(grad.abs().max()) > 0 else float((grad_t - grad).abs().max()),
            "tape_bytes": 4 * 6 * p.ncells * 8 * nsteps,
            "note": "checkpoint_every=0: the forward pass records every step's stage inputs "
                    "(device tape), the backward recomputes nothing"},
    }
    return line


def accuracy_main(args):
    """--workload accuracy: the mixed precision form against FP64 at the
    configured run lengths -- 2D Orszag-Tang (1e-3 rho noise) 1024^2 and
    4096^2 for 500 RK4 steps, the 3D stratified tube 256^3 for 1000 RK4
    steps: relative L2 distance per evolved field, and both forms' rates
    (CUDA events over the whole run).  Beside it, the sensitivity of the FP64
    solution itself: an FP64 run whose evolved state is rounded to float once,
    after step 10 (one rounding of the kind a float-storage form makes at
    every stage), against the plain FP64 run."""
    import numpy as np
    import torch
    from smaug_b200 import engine
    cases = [("ot", 1024, 500), ("ot", 4096, 500), ("tube", 256, 1000)]
    out = []
    for kind, n, nsteps in cases:
        states, ms = [], []
        for prec, rounded in ((0, False), (1, False), (0, True)):
            p, w, pos = (make_tube if kind == "tube" else make_case)(n, 1, prec)
            nevo = p.nvar - (4 if p.ndim == 2 else 5)
            e = engine.Engine(p, w, pos)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record()
            if rounded:
                e.step(10)
                st = e.state()
                st[:nevo] = st[:nevo].astype(np.float32).astype(np.float64)
                e.set_state(st)
                del st
                e.step(nsteps - 10)
            else:
                e.step(nsteps)
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
            states.append(e.state()[:nevo])
            e.close()
            del w, pos

        def rel(x):
            r = []
            for f in range(states[0].shape[0]):
                d = float(np.sqrt(np.sum((x[f] - states[0][f]) ** 2)))
                nrm = float(np.sqrt(np.sum(states[0][f] ** 2)))
                r.append(d / nrm if nrm > 0 else d)
            return r
        errs, sens = rel(states[1]), rel(states[2])
        cells = n ** (3 if kind == "tube" else 2)
        dims = "x".join([str(n)] * (3 if kind == "tube" else 2))
        out.append({"case": "%s %s, %d RK4 steps" % ("3D stratified tube" if kind == "tube" else
                                                     "2D Orszag-Tang", dims, nsteps),
                    "rel_l2_per_field": errs, "max": max(errs),
                    "fp64_rounded_once_at_step_10_rel_l2_per_field": sens,
                    "fp64_mcell_updates_per_s": cells * nsteps / (ms[0] / 1e3) / 1e6,
                    "mixed_mcell_updates_per_s": cells * nsteps / (ms[1] / 1e3) / 1e6})
        states = None
    line = {"metric": "mixed vs FP64 relative L2 per evolved field at the configured run length",
            "value": max(c["max"] for c in out[:2]), "unit": "relative L2 (2D cases)", "n_gpus": 1,
            "steps": None, "warmup": 0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 vs f32 storage", "data": "synthetic", "target": 1e-5,
            "config": {"workload": "Orszag-Tang 1024^2 and 4096^2 (500 steps), stratified tube 256^3 "
                                   "(1000 steps), seeded"}, "cases": out}
    print(json.dumps(line), flush=True)


def snapshots_main(args):
    """--workload snapshots: RK4 steps of a 1024^2 Orszag-Tang grid with a
    reference .out snapshot every 10 steps (the driver's cfgsavefrequency
    output, src/iosmaug.c:509-517), written synchronously (smaug_write_out)
    and asynchronously (smaug_write_out_async: copy queued on the stream,
    file written by a host thread while the engine steps).  Host wall clock
    over the whole loop, files included; value = the asynchronous steps/s."""
    import shutil
    import tempfile
    import torch
    from smaug_b200 import engine
    n = args.n if args.n is not None and args.n != WORKLOAD_N else 1024
    nsteps, every = 60, 10
    p, w, pos = make_case(n, 1, 0)
    out = tempfile.mkdtemp(prefix="smaug_snap_")
    res = {}
    try:
        for mode in ("sync", "async", "none"):
            e = engine.Engine(p, w, pos)
            e.step(args.warmup)
            t0 = time.perf_counter()
            for k in range(nsteps // every):
                e.step_async(every)
                path = os.path.join(out, "%s_%d.out" % (mode, k))
                if mode == "sync":
                    e.write_out(path, it=k, t=0.0)
                elif mode == "async":
                    e.write_out_async(path, it=k, t=0.0)
            if mode == "async":
                e.wait_writes()
            e.sync()
            torch.cuda.synchronize()
            res[mode] = time.perf_counter() - t0
            e.close()
        same = all(open(os.path.join(out, "sync_%d.out" % k), "rb").read() ==
                   open(os.path.join(out, "async_%d.out" % k), "rb").read() for k in range(nsteps // every))
        size = os.path.getsize(os.path.join(out, "sync_0.out"))
    finally:
        shutil.rmtree(out, ignore_errors=True)
    line = {"metric": "RK4 steps/s with a .out snapshot every %d steps" % every,
            "value": nsteps / res["async"], "unit": "steps/s", "n_gpus": 1, "steps": nsteps,
            "warmup": args.warmup, "ms_per_step": res["async"] / nsteps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "2D Orszag-Tang %dx%d, FP64 RK4, snapshot every %d steps" % (n, n, every),
                       "timing": "host wall clock over the loop, files written and closed"},
            "sync_steps_per_s": nsteps / res["sync"], "no_output_steps_per_s": nsteps / res["none"],
            "speedup_vs_sync": res["sync"] / res["async"], "bytes_per_snapshot": size,
            "files_identical": bool(same)}
    print(json.dumps(line), flush=True)


def max_over_ranks(ms, ws, device="cuda"):
    """The slowest rank's time: every rank takes part (the same collective in
    the same order on every rank); one rank returns its own value."""
    if ws <= 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        import datetime
        if args.impl != "reference":  # the reference arm runs on the host cores only
            torch.cuda.set_device(local)
        dist.init_process_group("nccl" if args.impl != "reference" else "gloo",
                                timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def cpu_sample(N=512, steps=1):
    """Oracle (the reference arithmetic on CPU, all host threads) on a
    bounded sample: `steps` RK4 steps of an N x N Orszag-Tang grid."""
    from oracle import pyoracle
    p, w, pos = make_case(N)
    run = pyoracle.OracleRun(p, w, pos)
    t0 = time.perf_counter()
    run.advance(steps)
    el = time.perf_counter() - t0
    return N * N * steps / el / 1e6, el, pyoracle.num_threads()


def reference_arm(args, ws, rank):
    if rank != 0:
        return
    from oracle import build
    build.build()
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    N = args.ref_sample
    for _ in range(args.warmup):
        cpu_sample(N, 1)
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        v, el, thr = cpu_sample(N, 1)
        vals.append(el)
    total = time.perf_counter() - t0
    value = N * N * args.steps / sum(vals) / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(vals) / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "2D Orszag-Tang %dx%d sample of the %dx%d workload, FP64, RK4"
                   % (N, N, WORKLOAD_N, WORKLOAD_N), "parallelism": "cpu",
                   "sample_cells": N * N},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": thr, "kind": "port",
                         "sample": "%d RK4 steps of a %dx%d Orszag-Tang grid per measured "
                                   "step; oracle/smaug_oracle.c (OpenMP)" % (1, N, N)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": total,
    }
    print(json.dumps(line), flush=True)


def reference_gpu_binary(timeout=240, name="ot1024t",
                         kind="reference binary built from source, its own per-step timer"):
    """Per-step time of the reference's own GPU binary (built from its
    sources by oracle/build_ref.py, Euler, 1024^2): Mcell-updates/s per
    Euler step from its own 'time total' lines, first 5 steps discarded.
    name="compat_ot1024t" times the same unchanged driver linked against the
    wrapper shim (libsmaug_compat2d.so), i.e. the reference's host loop
    driving this engine."""
    binp = os.path.join(ROOT, "oracle", "_ref", name, "smaug")
    if not os.path.exists(binp):
        return None
    import tempfile
    from smaug_b200 import formats
    from oracle import run_ref
    p, w, pos = make_case(1024)
    d = tempfile.mkdtemp(prefix="refbin_")
    ini = os.path.join(d, "in.ini")
    formats.write_ini(ini, w, pos)
    try:
        rc, times = run_ref.run(binp, ini, os.path.join(d, "run"), keep=set(), timeout=timeout)
    except Exception as e:  # noqa: BLE001
        return {"error": str(e)}
    if rc != 0 or len(times) < 8:
        return {"error": "rc=%s steps=%d" % (rc, len(times))}
    tt = [t for s, t in times]
    per = (tt[-1] - tt[4]) / (len(tt) - 5)
    v = 1024 * 1024 / per / 1e6
    # an RK4 step evaluates the spatial operator four times: the Euler rate / 4
    # is the reference's equivalent of this line's metric
    return {"value": v, "unit": "Mcell-updates/s per Euler step",
            "rk4_equivalent": {"value": v / 4, "unit": UNIT + " (4 operator evaluations per step)"},
            "ms_per_step": per * 1e3, "workload": "2D Orszag-Tang 1024x1024, FP64, Euler",
            "kind": kind}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ot", choices=["ot", "tube", "ensemble", "adjoint", "snapshots",
                                                        "accuracy"])
    ap.add_argument("--adj-steps", type=int, default=400)
    ap.add_argument("--obs-z", type=float, default=0.4e6,
                    help="height of the observed v_z row for --workload adjoint [m] (the "
                         "configured 3 Mm row is reported beside it)")
    ap.add_argument("--nruns", type=int, default=64)
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="default: fp64 (ot, tube; mixed reported beside it), mixed (ensemble)")
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--stencil-order", type=int, default=4, choices=[4, 6],
                    help="flux derivative order (6: the reference's USE_DORDER3 build)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--ref-sample", type=int, default=512)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--staging", type=int, default=0, choices=[0, 1, 2],
                    help="2D tile staging: 0 per-thread loads (default), 1 bulk tensor copies in a "
                         "persistent grid, 2 bulk tensor copies with a block per tile")
    ap.add_argument("--no-mixed", dest="mixed", action="store_false",
                    help="skip the mixed precision measurement")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.n is None:
        args.n = TUBE_N if args.workload == "tube" else WORKLOAD_N
    if args.precision == "mixed":
        args.mixed = False
    ws, rank, local = dist_setup(args)
    if args.precision is None:
        args.precision = "mixed" if args.workload == "ensemble" else "fp64"
    if args.workload == "ensemble" and args.impl != "reference":
        ensemble_main(args)
        return
    if args.workload == "adjoint" and args.impl != "reference":
        adjoint_main(args)
        return
    if args.workload == "snapshots" and args.impl != "reference":
        snapshots_main(args)
        return
    if args.workload == "accuracy" and args.impl != "reference":
        accuracy_main(args)
        return
    if args.impl == "reference":
        reference_arm(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import numpy as np
    import torch
    from smaug_b200 import engine

    torch.cuda.set_device(local)
    N = args.n
    p, w, pos, ncell_int, desc = workload(args, seed=1 + rank)
    eng = engine.Engine(p, w, pos)
    # a dedicated stream: the engine launches on it, the events are recorded on it
    stream = torch.cuda.Stream()
    assert stream.cuda_stream != 0
    eng.set_stream(stream.cuda_stream)
    if args.staging:
        eng.set_staging(args.staging)
    alg_bytes = alg_bytes_per_cell_step(p.ndim)

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    # warm-up
    eng.step_async(args.warmup)
    eng.sync()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        eng.step_async(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    eng.sync()
    barrier()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, ws)
    value = ncell_int * args.steps * ws / (ms_max / 1e3) / 1e6
    launches = 4 * args.steps
    ref_state = eng.state() if args.mixed else None

    # e2e: host buffers through the C ABI, pinned memory, copies in the timed region
    nvar = p.nvar
    host = torch.empty((nvar,) + p.shape, dtype=torch.float64, pin_memory=True).numpy()
    eng.state(out=host)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    nevo = 2 + 2 * p.ndim
    for _ in range(args.e2e_steps):
        eng.set_state(host)      # H2D of the evolved fields
        eng.step(1)
        eng.fields(0, nevo, out=host[:nevo])   # D2H of the step's result (the evolved fields)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), ws)
    e2e_val = ncell_int * args.e2e_steps * ws / (e2e_ms / 1e3) / 1e6
    h2d = (2 + 2 * p.ndim) * p.ncells * 8
    d2h = nevo * p.ncells * 8
    # the other tile stagings of the 2D kernel on the same engine (bitwise the
    # same arithmetic), timed like the headline
    staging = None
    if p.ndim == 2 and eng.staging()[1]:
        staging = {"selected": args.staging, "ms_per_step": {}}
        names = {0: "per-thread loads", 1: "bulk tensor copies, persistent grid",
                 2: "bulk tensor copies, a block per tile"}
        for mode in (0, 1, 2):
            eng.set_staging(mode)
            eng.step_async(args.warmup)
            s0 = torch.cuda.Event(enable_timing=True)
            s1 = torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            eng.step_async(args.steps)
            s1.record(stream)
            torch.cuda.synchronize()
            eng.sync()
            staging["ms_per_step"][names[mode]] = max_over_ranks(s0.elapsed_time(s1), ws) / args.steps
        eng.set_staging(args.staging)
    eng.close()

    # the mixed precision form on the same workload: same warm-up and timed
    # steps, its state compared with the FP64 state after the same steps
    mixed = None
    if args.mixed:
        from smaug_b200 import params as P
        pm = P.SmaugParams.from_buffer_copy(p)
        pm.precision = P.PREC_MIXED
        em = engine.Engine(pm, w, pos)
        em.set_stream(stream.cuda_stream)
        if args.staging and em.staging()[1]:
            em.set_staging(args.staging)
        em.step_async(args.warmup)
        em.sync()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        em.step_async(args.steps)
        m1.record(stream)
        torch.cuda.synchronize()
        em.sync()
        barrier()
        mms = max_over_ranks(m0.elapsed_time(m1), ws)
        mst = em.state()
        em.close()
        nevo = 2 + 2 * p.ndim
        errs = []
        for f in range(nevo):
            d = float(np.sqrt(np.sum((mst[f] - ref_state[f]) ** 2)))
            n = float(np.sqrt(np.sum(ref_state[f] ** 2)))
            errs.append(d / n if n > 0 else d)
        mval = ncell_int * args.steps * ws / (mms / 1e3) / 1e6
        mbytes = alg_bytes_mixed(p.ndim)
        peak_m, _ = peaks()
        mach = mbytes * ncell_int * args.steps / (mms / 1e3) / 1e9
        mixed = {"value": mval, "unit": UNIT, "ms_per_step": mms / args.steps,
                 "speedup_vs_fp64": mval / value, "dtype": "f32 storage + hyperdiffusion, f64 rest",
                 "rel_l2_vs_fp64": {"steps": args.warmup + args.steps, "max": max(errs),
                                    "per_field": errs},
                 "roofline": roofline_block(p.ndim, "mixed", mbytes, ncell_int, args.steps, mms, peak_m,
                                            peaks()[1]),
                 "fp64_roofline": fp64_roofline(p.ndim, "mixed", ncell_int, args.steps, mms)}

    if rank == 0:
        peak, pk_kind = peaks()
        state_gb = (2 + 2 * p.ndim) * p.ncells * 8 / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc,
                       "interior_cells": ncell_int, "integrator": "rk4", "precision": "fp64",
                       "stencil_order": args.stencil_order,
                       "parallelism": "replicas" if ws > 1 else "single-gpu",
                       "l2": "state %.2f GB per buffer > 126 MB L2, no flush" % state_gb},
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": args.e2e_steps,
                    "path": "smaug_set_state + smaug_step + smaug_get_fields (evolved fields), pinned host buffers",
                    "gpu_launches_per_step": 4 + 2},
            "gpu_launches": launches,
            "roofline": roofline_block(p.ndim, args.precision, alg_bytes, ncell_int, args.steps, ms,
                                       peak, pk_kind),
            "fp64_roofline": fp64_roofline(p.ndim, args.precision, ncell_int, args.steps, ms_max),
            "clocks": clk.summary(),
            "mixed": mixed,
            "staging": staging,
        }
        if ws == 1 and not args.no_cpu_baseline and args.workload == "ot":
            os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
            v, el, thr = cpu_sample(args.ref_sample, 1)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": thr, "kind": "port",
                                    "sample": "1 RK4 step of a %dx%d Orszag-Tang grid (%.1f s), "
                                              "oracle/smaug_oracle.c, OpenMP" % (
                                                  args.ref_sample, args.ref_sample, el)}
        if ws == 1 and not args.no_ref_gpu and args.workload == "ot":
            line["reference_gpu"] = reference_gpu_binary()
            line["reference_driver_on_engine"] = reference_gpu_binary(
                name="compat_ot1024t",
                kind="the reference's unchanged driver (src/iosmaug.c) linked against "
                     "libsmaug_compat2d.so, its own per-step timer")
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
