#!/usr/bin/env python
"""Benchmark of the per-time-step hot path: cell-steps/s on the 256^3 ACDI
droplet workload (64 droplets, density ratio 1000, random divergence-free
initial velocity), FP64 drop-in form, one GPU per process.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

N > 1 runs under torchrun (one process per GPU, NCCL for the barrier and the
max-over-ranks timing).  The case does not shard across GPUs in this build:
each rank advances its own replica of the workload (weak scaling, no
data-path collective).  `--impl reference` times the CPU restatement of the
reference's algorithm (the reference itself needs a Fortran/MPI/FFTW build
that this machine cannot make) on the host cores, rank 0 only.

Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cans-fizzy_b200"))

METRIC = "cell-steps/s at 256^3 ACDI, mixed vs FP64 at stated error; ensemble cases/s"
WORKLOAD = ("droplets_acdi: 256^3 cells, unit box, periodic x,y, no-slip z walls, 64 droplets R~U[0.03,0.06] "
            "(seeded rejection sampler), rho 1000/1, mu 100/1, sigma 1, g 1, ACDI, random divergence-free "
            "u0 (|k|<=4, rms 0.1); AB2 step with FFT Poisson solve")
DATA = "synthetic (seeded generator, numpy default_rng(2026)); no dataset"

# The other configurations of the benchmark matrix (--config); the default,
# c3a, is the metric's own configuration above.
CONFIGS = {
    "c1": ("rising_bubble_3d", "rising bubble 64x64x128, domain 1x1x2, periodic x,y, no-slip z walls, bubble D 0.5, "
                               "rho 1000/100, mu 10/1, sigma 24.5, g 0.98, ACDI, fluid at rest"),
    "c3b": ("droplets_thinc", "droplets_thinc: 512x512x256 cells, box 2x2x1, 64 droplets R~U[0.03,0.06], rho 1000/1, "
                              "mu 100/1, sigma 1, g 1, THINC/QQ (beta 1), random divergence-free u0"),
    "c5": ("shear_stretched", "shear_stretched: 512x256x256, tanh-stretched z (gr 1.5), Poiseuille mean 1 driven by "
                              "the laminar pressure gradient, 1% perturbation, 200 droplets R~U[0.04,0.08], "
                              "rho 10/1, mu 1/1, sigma 0.5, ACDI"),
}

# Algorithmic bytes per cell of each profiled stage (one read of every input
# point, one write of every output point; halo and neighbour re-reads are
# not counted).  FP64 drop-in:
STAGE_BYTES = {
    # psi, phi, u, v, w, normx/y/z, history (r) + psi_new, history, fx, fy, fz (w)
    "phase_transport": 8 * (9 + 5),
    "cmpt_phi": 8 * 2,
    "youngs": 8 * (1 + 4),
    # u,v,w, psi, psio, fx,fy,fz, p, po, kappa, 3 histories (r) + 3 histories, u,v,w (w)
    "momentum": 8 * (14 + 6),
    "poisson_x_fwd_fillps": 8 * (3 + 1),
    "poisson_y_fwd": 8 * 2,
    "poisson_z_solve": 8 * 2,
    "poisson_y_bwd": 8 * 2,
    "poisson_x_bwd": 8 * 2,
    # correc: phi, u, v, w (r) + u, v, w (w); updatep: p (r) + p_new (w)
    "correc_updatep": 8 * (1 + 6 + 2),
    "gamma_chkdt_chkdiv": 8 * 3,
    # scalar (_SCALAR): s, psi, psio, u, v, w, fx, fy, fz, history (r) + s_new, history (w)
    "scalar": 8 * (10 + 2),
}
# mixed form: state u, v, w, p, psi FP64; phi, normals, kappa, fluxes, histories
# and the spectral work buffer FP32
STAGE_BYTES_MIXED = {
    "phase_transport": 8 * 5 + 4 * 5 + 8 + 4 * 4,
    "cmpt_phi": 8 + 4,
    "youngs": 4 * (1 + 4),
    "momentum": 8 * 7 + 4 * 7 + 4 * 3 + 8 * 3,
    "fillps": 8 * 4,
    "poisson_f32": (8 + 4) + 4 * 2 * 3 + (4 + 8),
    # correc: phi, u, v, w (r) + u, v, w (w); updatep: p (r) + p_new (w)
    "correc_updatep": 8 * (1 + 6 + 2),
    "gamma_chkdt_chkdiv": 8 * 3,
}
B_ALG_STEP = 232  # bytes per cell-step: 19 state accesses + 10 Poisson-pass accesses (FP64)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="cansfz", choices=["cansfz", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=240.0,
                    help="upper bound on the seconds of timed CPU work (reference arm)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--grid", type=int, default=256, help="cube size of the droplet workload (profiling runs)")
    ap.add_argument("--form", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--sweeps", type=int, default=-1,
                    help="refinement sweeps of the mixed form's FP32 Poisson solve (-1: the solve in FP64)")
    ap.add_argument("--config", default="c3a", choices=["c3a", "c1", "c3b", "c5", "c2"],
                    help="benchmark-matrix configuration (c3a: the metric's 256^3 ACDI case; c2: Poisson only)")
    ap.add_argument("--scalar-steps", type=int, default=50,
                    help="steps of the scalar-transport leg (0: skip)")
    ap.add_argument("--ensemble-steps", type=int, default=100,
                    help="steps per case of the batched-ensemble measurement (0: skip)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default launch plan instead of the autotuned one")
    ap.add_argument("--no-mixed-leg", dest="mixed_leg", action="store_false",
                    help="skip the mixed-form leg of an FP64 run")
    ap.add_argument("--accuracy-steps", type=int, default=50,
                    help="mixed form: steps of the error check against the FP64 form (0: skip)")
    return ap.parse_args()


def select_workload(args):
    """(params, fields, workload description) of the configuration the run
    measures; the GPU arm and the reference arm build it identically."""
    from cansfz import workloads as W

    if args.config in CONFIGS:
        builder, workload = CONFIGS[args.config]
        p, fields = W.BUILDERS[builder]()
    elif args.grid == 256:
        workload = WORKLOAD
        p, fields = W.droplets_acdi(seed=2026)
    else:
        p, fields = W.droplets((args.grid,) * 3, (1.0, 1.0, 1.0), False, seed=2026)
        workload = f"droplets_acdi at {args.grid}^3 (profiling size)"
    return p, fields, workload


def run_config(args, p, workload, world):
    """The `config` object of the JSON line: what the workload is, not what a
    run measured, so that both arms print the same object."""
    nx, ny, nz = p.n
    hbytes = 8 * (nx + 2) * (ny + 2) * (nz + 2)
    return {"workload": workload, "config": args.config, "grid": [nx, ny, nz],
            "form": "fp64 (drop-in)" if args.form == "fp64" else
                    ("mixed (FP32 stencils, fluxes, curvature and histories; FP64 state, AB2 accumulation, "
                     "reductions and Poisson solve)" if args.sweeps < 0 else
                     f"mixed (FP32 stencils and transforms, FP64 state, AB2 accumulation and reductions, "
                     f"{args.sweeps} FP64-residual refinement sweeps)"),
            "parallelism": "replicas" if world > 1 else "single",
            "l2": (f"inputs larger than L2 (each FP64 field {hbytes / 1e6:.0f} MB > 126 MB; ~28 fields resident), "
                   "no flush needed" if hbytes > 126e6 else
                   f"profiling size: each FP64 field {hbytes / 1e6:.1f} MB < 126 MB L2, no flush")}


def plan_cache():
    """The autotuner's cache file (one line per grid/form/GPU key)."""
    d = os.environ.get("CANSFZ_PLAN_CACHE_DIR", os.path.join(os.path.expanduser("~"), ".cache", "cansfz"))
    os.makedirs(d, exist_ok=True)
    return os.path.join(d, "plans.txt")


def plan_dict(q, report):
    return {"phase_slots": q.phase_slots, "momentum_slots": q.momentum_slots,
            "zsolve": "partitioned tiles" if q.zsolve == 0 else "one column per thread",
            "fp32_transforms": "tcgen05 GEMM" if q.fp32_transforms == 0 else "FFT",
            "tile_staging": "TMA" if q.tile_tma else "cp.async",
            "ghost_images": "written by the producing kernels" if q.ghost_images else "fill stages",
            "line_transforms": "two register passes" if q.line_transforms == 0 else "warp per line / Stockham",
            "tuned_ms_per_step": q.ms_per_step, "report": report}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback (MEASURED_PEAKS.json absent: an earlier copy measurement on this pool)"


class Clocks:
    """nvidia-smi sampling of the SM clock and throttle reasons (200 ms)."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.p = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, smax, power, reasons = [], [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in out.splitlines():
            cols = [c.strip() for c in line.split(",")]
            if len(cols) < 9:
                continue
            if self.uuid and self.uuid not in cols[0]:
                continue
            try:
                sm.append(float(cols[1]))
                smax.append(float(cols[2]))
                power.append(float(cols[3]))
            except ValueError:
                continue
            for nm, val in zip(names, cols[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        busy = [s for s, p in zip(sm, power) if p > 0.3 * max(power)] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": max(smax), "samples": len(sm),
                "power_w_max": max(power), "reasons": sorted(reasons)}


def dist_setup(n_gpus: int):
    """One process per GPU under torchrun (cansfz/replicas.py); NCCL between GPU ranks."""
    from cansfz import replicas

    return replicas.setup()


def allreduce_max(x: float, world: int) -> float:
    from cansfz import replicas

    return replicas.max_over_ranks(x, world)


def barrier(world: int):
    from cansfz import replicas

    replicas.barrier(world)


def cpu_run(p, fields, budget_s: float, warmup: int = 1, max_steps: int = 1000):
    """The CPU restatement (oracle/) on the same workload: warm-up steps, then
    timed steps until `budget_s` of CPU work; returns (cell-steps/s, steps, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    threads = O.set_threads(os.cpu_count() or 1)
    c = O.Case(p)
    for name, a in zip(("u", "v", "w", "p", "psi"), fields):
        c.set(name, a)
    c.prepare()
    if warmup:
        c.step(warmup)
    n = 0
    t0 = time.perf_counter()
    while n < max_steps:
        c.step(1)
        n += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    cells = p.ng[0] * p.ng[1] * p.ng[2]
    return cells * n / dt, n, threads, dt


def mixed_accuracy(p, fields, nsteps):
    """Relative errors of the mixed form against the FP64 form (itself pinned to
    the oracle) after `nsteps` steps from the same state: max|a-b|/max|b| for
    u, v, w, psi and mean-free p; phase-mass drift and max divergence of both."""
    import numpy as np

    from cansfz import case as C

    res = {}
    runs = {}
    for form in (0, 1):
        q = p.copy()
        q.form = form
        c = C.Case(q)
        c.set_fields(*fields)
        c.prepare()
        m0 = c.diag().mass12[0]
        rc = c.step(nsteps)
        if rc != 0:
            raise RuntimeError(f"accuracy run (form {form}) failed with status {rc}")
        d = c.diag()
        runs[form] = {nm: c.get(nm) for nm in ("u", "v", "w", "p", "psi")}
        res["fp64" if form == 0 else "mixed"] = {"mass_drift_rel": abs(d.mass12[0] - m0) / m0, "divmax": d.divmax}
        c.close()
    err = {}
    for nm in ("u", "v", "w", "psi", "p"):
        a, b = runs[1][nm][1:-1, 1:-1, 1:-1], runs[0][nm][1:-1, 1:-1, 1:-1]
        if nm == "p":
            a, b = a - a.mean(), b - b.mean()
        err[nm] = float(np.abs(a - b).max() / np.abs(b).max())
    res["steps"] = nsteps
    res["rel_err_max"] = err
    return res


def mixed_leg(args, p0, fields, fp64_ms_step):
    """The mixed-precision form on the same workload: W warm-up and K timed
    graph-launched steps (device time, CUDA events on the case's stream),
    its speed-up over the FP64 step, and its error against the FP64 form
    after `--accuracy-steps` steps from the same state."""
    import torch

    from cansfz import case as C

    q = p0.copy()
    q.form = 1
    q.refine_sweeps = args.sweeps
    c = C.Case(q)
    c.set_fields(*fields)
    c.prepare()
    plan, plan_report = c.autotune(plan_cache()) if args.autotune else (c.plan(), "default plan")
    if c.step(args.warmup) != 0:
        raise RuntimeError("mixed warm-up failed")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(c.stream)
    rc = c.step(args.steps)
    ev1.record(c.stream)
    torch.cuda.synchronize()
    if rc != 0:
        raise RuntimeError(f"mixed steps failed with status {rc}")
    ms = ev0.elapsed_time(ev1) / args.steps
    c.close()
    nx, ny, nz = p0.n
    out = {"value": nx * ny * nz / (ms * 1e-3), "unit": "cell-steps/s", "ms_per_step": ms,
           "steps": args.steps, "warmup": args.warmup, "speedup_vs_fp64": fp64_ms_step / ms,
           "refine_sweeps": args.sweeps, "plan": plan_dict(plan, plan_report),
           "form": ("FP32 stencils, fluxes, curvature and AB2 histories; FP64 state, AB2 accumulation, reductions "
                    "and Poisson solve") if args.sweeps < 0 else
                   (f"FP32 stencils and transforms, FP64 state, AB2 accumulation and reductions, {args.sweeps} "
                    "FP64-residual refinement sweeps")}
    if args.accuracy_steps > 0:
        out["accuracy_vs_fp64"] = mixed_accuracy(q, fields, args.accuracy_steps)
    return out


def scalar_bench(p0, fields, nsteps, peak):
    """The same workload with the scalar transport and Boussinesq buoyancy on
    (_SCALAR, _BOUSSINESQ_BUOYANCY: s Dirichlet 1/0 at the z walls, Couette
    start, rho*cp and k of both phases unequal): device time per step of
    the graph-launched step, and the scalar stage (k_scal_step) against its
    algorithmic bytes (96 B per cell) from the stage profile."""
    import torch

    from cansfz import case as C
    from cansfz import lib as _L

    p = p0.copy()
    p.scalar, p.boussinesq = 1, 1
    p.cbcsca = b"PPPPDD"
    p.bcsca[:] = [0.0, 0.0, 0.0, 0.0, 1.0, 0.0]
    p.ka12[:] = [1e-3, 2e-3]
    p.cp12[:] = [1.5, 1.0]
    case = C.Case(p)
    case.set_fields(*fields)
    case.initscal("cou")
    case.prepare()
    stream = torch.cuda.current_stream()
    if case.step(3) != 0:
        raise RuntimeError("scalar warm-up failed")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    rc = case.step(nsteps)
    ev1.record(stream)
    torch.cuda.synchronize()
    if rc != 0:
        raise RuntimeError(f"scalar steps failed with status {rc}")
    ms_step = ev0.elapsed_time(ev1) / nsteps
    nprof = 3
    buf = (_L.ct.c_double * 64)()
    nst = _L.ct.c_int(0)
    names = _L.ct.create_string_buffer(4096)
    _L.check(case.lib.cansfz_profile_stages(case.h, nprof, buf, 64, _L.ct.byref(nst), names, 4096), "profile")
    stage = {nm: buf[q] / nprof for q, nm in enumerate(names.value.decode().split(","))}
    cells = p.ng[0] * p.ng[1] * p.ng[2]
    ach = STAGE_BYTES["scalar"] * cells / (stage["scalar"] * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        if "scalar" in tj:
            traffic = tj["scalar"]["bytes_per_cell"] * cells
    case.close()
    return {"ms_per_step": ms_step, "steps": nsteps, "scalar_stage_ms": stage["scalar"],
            "bc_scalar_ms": stage.get("bc_scalar"), "momentum_ms": stage.get("momentum"),
            "roofline": {"kernel": "k_scal_step", "bound": "hbm", "bytes_per_cell": STAGE_BYTES["scalar"],
                         "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "traffic": traffic},
            "what": "the headline workload with _SCALAR and _BOUSSINESQ_BUOYANCY on; device time, graph-launched"}


def ensemble_bench(nsteps, warmup, form, tune=True):
    """The batched-ensemble configuration: 64 independent rising-bubble cases,
    `nsteps` steps each, run (a) one case at a time (each case's own graph,
    cansfz_step) and (b) batched (cansfz_ensemble_step: one graph launch per
    step for all cases), from the same initial states.  cases/s = completed
    case-runs per second, wall clock around synchronised work."""
    import torch

    from cansfz import case as C
    from cansfz import workloads as W

    specs = W.ensemble_cases(seed=4)

    reports = {}

    def build():
        cs = []
        for p, f in specs:
            q = p.copy()
            q.form = form
            c = C.Case(q, own_stream=True)
            c.set_fields(*f)
            c.prepare()
            if tune:
                # one timing per grid shape (the cache holds the rest)
                pl, rep = c.autotune(plan_cache())
                reports.setdefault(f"{q.ng[0]}x{q.ng[1]}x{q.ng[2]}", plan_dict(pl, rep))
            cs.append(c)
        return cs

    seq = build()
    for c in seq:  # warm-up: graph capture and first steps
        if c.step(warmup) != 0:
            raise RuntimeError("ensemble warm-up failed")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for c in seq:
        rc = c.step(nsteps)
        if rc != 0:
            raise RuntimeError(f"sequential ensemble case failed with status {rc}")
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    seq_state = [c.get("psi") for c in seq[:4]]
    for c in seq:
        c.close()
    bat = build()
    ens = C.Ensemble(bat)
    rc, _ = ens.step(warmup)
    if rc != 0:
        raise RuntimeError("batched ensemble warm-up failed")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc, sts = ens.step(nsteps)
    torch.cuda.synchronize()
    t_bat = time.perf_counter() - t0
    if rc != 0:
        raise RuntimeError(f"batched ensemble failed with statuses {sts}")
    # the batched run computes exactly what the one-at-a-time run computes
    same = all(float(abs(a - c.get("psi")).max()) == 0.0 for a, c in zip(seq_state, bat[:4]))
    ens.close()
    cells = sum(int(p.n[0] * p.n[1] * p.n[2]) for p, _ in specs)
    for c in bat:
        c.close()
    n = len(specs)
    return {"cases": n, "steps_per_case": nsteps, "warmup": warmup, "form": "fp64" if form == 0 else "mixed",
            "cells_total": cells,
            "cases_per_s_batched": n / t_bat, "cases_per_s_sequential": n / t_seq,
            "speedup": t_seq / t_bat, "cell_steps_per_s_batched": cells * nsteps / t_bat,
            "batched_equals_sequential": bool(same),
            "plans": reports,
            "what": "64 rising-bubble cases (seed 4; 32 2-D 64x128..256x512, 32 3-D 32^3..96x96x192); "
                    "wall clock around synchronised work"}


def gpu_arm(args):
    import numpy as np
    import torch

    from cansfz import case as C
    from cansfz import lib as _L
    from cansfz import workloads as W

    rank, world, local = dist_setup(args.gpus)
    p, fields, workload = select_workload(args)
    if args.form == "mixed":
        p.form = 1
        p.refine_sweeps = args.sweeps
    nx, ny, nz = p.n
    cells = nx * ny * nz
    case = C.Case(p)
    case.set_fields(*fields)
    case.prepare()
    # launch plan: timed on a copy of the case, cached per grid/form/GPU
    plan, plan_report = case.autotune(plan_cache()) if args.autotune else (case.plan(), "default plan")
    rc = case.step(args.warmup)
    if rc != 0:
        raise RuntimeError(f"warm-up step failed with status {rc}")
    stream = case.stream
    kps = _L.ct.c_int(0)
    _L.check(case.lib.cansfz_kernels_per_step(case.h, _L.ct.byref(kps)), "kernels_per_step")
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(torch.cuda.current_device()).uuid)
    except Exception:
        pass
    # ---- timed region: K graph-launched steps, device time, max over ranks
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    clk = Clocks(uuid)
    ev0.record(stream)
    rc = case.step(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = clk.stop()
    if rc != 0:
        raise RuntimeError(f"timed steps failed with status {rc}")
    ms = allreduce_max(ev0.elapsed_time(ev1), world)
    ms_step = ms / args.steps
    value = cells * args.steps * world / (ms / 1e3)
    d = case.diag()
    # ---- stage profile (events between stages, outside the graph)
    nprof = 5
    buf = (_L.ct.c_double * 64)()
    nst = _L.ct.c_int(0)
    names = _L.ct.create_string_buffer(4096)
    _L.check(case.lib.cansfz_profile_stages(case.h, nprof, buf, 64, _L.ct.byref(nst), names, 4096), "profile")
    stage_names = names.value.decode().split(",")
    stage_ms = {nm: buf[q] / nprof for q, nm in enumerate(stage_names)}
    tot = sum(stage_ms.values())
    table = STAGE_BYTES if args.form == "fp64" else STAGE_BYTES_MIXED
    heavy = [s for s in stage_ms if s in table]
    dom = max(heavy, key=lambda s: stage_ms[s])
    peak, peak_kind = measured_peaks()
    bytes_launch = table[dom] * cells
    achieved = bytes_launch / (stage_ms[dom] * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        key = dom if args.form == "fp64" else dom + ":mixed"
        if key in tj:
            traffic = tj[key]["bytes_per_cell"] * cells
    out = {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else
        ("f64 state, momentum and Poisson / f32 phase field" if args.sweeps < 0 else
         "f64 state and momentum / f32 phase field and transforms"),
        "data": DATA,
        "config": run_config(args, p, workload, world),
        "run": {"final_time": d.time, "final_dt": d.dt, "divmax": d.divmax},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "bytes_per_launch": bytes_launch, "traffic": traffic,
                     "step_frac": (B_ALG_STEP * cells / (ms_step * 1e-3) / 1e9) / peak},
        "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "stage_share": {k: round(v / tot, 4) for k, v in stage_ms.items()},
        "gpu_launches": int(kps.value) * args.steps,
        "clocks": clocks,
        "plan": plan_dict(plan, plan_report),
    }
    # ---- the same workload with the scalar transport
    if world == 1 and args.config == "c3a" and args.form == "fp64" and args.scalar_steps > 0:
        out["scalar"] = scalar_bench(p, fields, args.scalar_steps, peak)
        out["scalar"]["overhead"] = out["scalar"]["ms_per_step"] / ms_step - 1.0
    # ---- batched ensemble of independent small cases
    if world == 1 and args.ensemble_steps > 0 and args.config == "c3a":
        out["ensemble"] = ensemble_bench(args.ensemble_steps, 3, 0 if args.form == "fp64" else 1, args.autotune)
    # ---- mixed form: error against the FP64 form after the same steps from the same state
    if args.form == "mixed" and args.accuracy_steps > 0:
        out["accuracy_vs_fp64"] = mixed_accuracy(p, fields, args.accuracy_steps)
    # ---- the metric's second leg: the mixed form beside the FP64 headline
    if world == 1 and args.form == "fp64" and args.mixed_leg:
        out["mixed"] = mixed_leg(args, p, fields, ms_step)
    # ---- end to end through the C ABI with pinned host buffers
    if not args.no_e2e:
        hshape = tuple(x + 2 for x in p.n)
        pin = [torch.empty(int(np.prod(hshape)), dtype=torch.float64).pin_memory() for _ in range(5)]
        for t, a in zip(pin, fields):
            t.copy_(torch.from_numpy(np.ascontiguousarray(a.reshape(-1, order="F"))))
        ptrs = [_L.ct.c_void_p(t.data_ptr()) for t in pin]
        e2e_case = C.Case(p)
        if args.autotune:
            e2e_case.autotune(plan_cache())  # the headline case's cached plan
        ksteps = args.steps
        diag = _L.Diag()
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _L.check(e2e_case.lib.cansfz_set_fields(e2e_case.h, *ptrs, 0), "set_fields")
        _L.check(e2e_case.lib.cansfz_prepare(e2e_case.h), "prepare")
        for _ in range(ksteps):
            rc = e2e_case.lib.cansfz_step(e2e_case.h, 1)
            _L.check(e2e_case.lib.cansfz_get_status(e2e_case.h, _L.ct.byref(diag)), "get_status")
            if rc:
                break
        _L.check(e2e_case.lib.cansfz_get_diag(e2e_case.h, _L.ct.byref(diag)), "get_diag")
        _L.check(e2e_case.lib.cansfz_get_fields(e2e_case.h, *ptrs, 0), "get_fields")
        torch.cuda.synchronize()
        te = allreduce_max(time.perf_counter() - t0, world)
        fb = 8 * int(np.prod(hshape))
        out["e2e"] = {"value": cells * ksteps * world / te, "unit": "cell-steps/s",
                      "h2d_bytes_per_step": 5 * fb / ksteps,
                      "d2h_bytes_per_step": (5 * fb + (ksteps + 1) * _L.ct.sizeof(_L.Diag)) / ksteps,
                      "what": "set_fields from pinned host, prepare, K x (cansfz_step(1) + cansfz_get_status: "
                              "time, dt, Gamma, status to the host every step), cansfz_get_diag (phase masses) "
                              "and get_fields to pinned host at the end; wall clock, max over ranks"}
        e2e_case.close()
    # ---- CPU baseline (rank 0, N = 1)
    if world == 1 and not args.no_cpu_baseline:
        v, n, thr, dt = cpu_run(p, fields, budget_s=15.0, warmup=1, max_steps=20)
        out["cpu_baseline"] = {"value": v, "unit": "cell-steps/s", "cores": thr, "kind": "port",
                               "sample": f"{n} steps of the same {nx}x{ny}x{nz} workload after 1 warm-up step "
                                         f"({dt:.1f} s), oracle/ C++ OpenMP restatement"}
    case.close()
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        from cansfz import replicas

        replicas.teardown(world)


def reference_arm(args):
    """The reference's algorithm on the host cores: the C++ OpenMP restatement
    in oracle/ (the reference itself is Fortran + MPI + FFTW, which this
    machine cannot build), W warm-up steps then K timed steps of the same
    workload and `config` as the GPU arm.  libcansfz is never loaded here:
    the workload's z grid comes from the oracle's initgrid."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from cansfz import init

    init.use_initgrid(O.lib().orc_initgrid)
    if args.config == "c2":
        print(json.dumps({"impl": "reference", "unavailable": "the Poisson-only configuration has no CPU arm"}))
        return
    p, fields, workload = select_workload(args)
    v, n, thr, dt = cpu_run(p, fields, budget_s=args.cpu_budget, warmup=args.warmup, max_steps=max(args.steps, 1))
    nx, ny, nz = p.n
    out = {"metric": METRIC, "value": v, "unit": "cell-steps/s", "n_gpus": world, "steps": n, "warmup": args.warmup,
           "ms_per_step": 1e3 * dt / n, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": DATA, "impl": "reference",
           "config": run_config(args, p, workload, world),
           "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": thr, "kind": "port",
                            "sample": f"{n} of the requested {args.steps} steps after {args.warmup} warm-up steps "
                                      f"(time budget {args.cpu_budget:.0f} s) of the {nx}x{ny}x{nz} workload in FP64: "
                                      "the reference is Fortran+MPI+FFTW and cannot be built here, so its CPU path "
                                      "runs as the C++ OpenMP restatement in oracle/"},
           "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def poisson_arm(args):
    """Configuration c2: the pressure solve alone at 256^3 (PPPPNN, RHS ~ N(0,1)
    with the mean removed): the FP64 solve and the FP32 solve with 0-3 FP64
    residual refinement sweeps; solves/s (device time of K solves, CUDA
    events) and, per sweep count, the 7-point residual (L2, Linf, relative to
    the RHS) and the error against the FP64 solution (mean removed)."""
    import numpy as np
    import torch

    from cansfz import case as C
    from cansfz import workloads as W

    dist_setup(1)
    p, rhs = W.poisson_rhs(256, 2026)
    g = C.Case(p)
    src = g.field(rhs)
    k = max(args.steps // 10, 3)

    def timed(fn):
        for _ in range(2):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(g.stream)
        for _ in range(k):
            fn()
        e1.record(g.stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    ref = g.field(rhs)
    g.call("solver", ref)
    a64 = ref.get()[1:-1, 1:-1, 1:-1]
    a64 = a64 - a64.mean()
    work = g.field(rhs)
    ms64 = timed(lambda: g.call("solver", work))
    r = g.field()
    out = g.field()
    rin = rhs[1:-1, 1:-1, 1:-1]
    res = {}
    # the FP32 solve with its x/y transforms as split-BF16 GEMMs on the tensor
    # cores, and with the shared-memory FFTs (fp32_transforms = 1)
    pf = p.copy()
    pf.fp32_transforms = 1
    gf = C.Case(pf)
    srcf, outf = gf.field(rhs), gf.field()

    def timed_f(fn):
        for _ in range(2):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(gf.stream)
        for _ in range(k):
            fn()
        e1.record(gf.stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    for sw in range(4):
        ms_fft = timed_f(lambda: gf.call("solver_refined", srcf, outf, sw))
        ms = timed(lambda: g.call("solver_refined", src, out, sw))
        b = out.get()[1:-1, 1:-1, 1:-1]
        b = b - b.mean()
        g.call("poisson_residual", src, out, r)
        rr = r.get()[1:-1, 1:-1, 1:-1]
        res[str(sw)] = {"ms_per_solve": ms, "solves_per_s": 1e3 / ms, "ms_per_solve_fft_transforms": ms_fft,
                        "residual_l2_rel": float(np.linalg.norm(rr) / np.linalg.norm(rin)),
                        "residual_linf_rel": float(np.abs(rr).max() / np.abs(rin).max()),
                        "err_vs_fp64_rel": float(np.abs(b - a64).max() / np.abs(a64).max())}
    print(json.dumps({"metric": "Poisson solves/s at 256^3 (PPPPNN)", "value": 1e3 / ms64, "unit": "solves/s",
                      "n_gpus": 1, "steps": k, "warmup": 2, "ms_per_step": ms64, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
                      "config": {"workload": "poisson_256: 256^3 uniform, periodic x,y, Neumann z, RHS ~ N(0,1) "
                                             "(seed 2026), mean removed", "config": "c2"},
                      "fp32_refined": res,
                      "fp32_transforms": "x/y as split-BF16 GEMMs on tcgen05 (ms_per_solve); shared-memory FFTs "
                                         "(ms_per_solve_fft_transforms)"}), flush=True)
    g.close()
    gf.close()


def main():
    args = parse_args()
    if args.impl == "reference":
        reference_arm(args)
    elif args.config == "c2":
        poisson_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
