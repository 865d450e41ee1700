"""Benchmark: fully-implicit oil-water timesteps on the 1.12M-cell
channelised model (60 x 220 x 85 cells of 6.1 x 3.05 x 0.61 m), metric
cell-Newton-iterations/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One "step" is one backward-Euler timestep (10 days) solved by Newton with the
device CPR-GMRES; consecutive steps continue the same schedule.  `value`
counts cells x Newton iterations over the timed steps divided by the device
time (CUDA events, max over ranks); `e2e` repeats the timed steps through the
public `GpuOilWaterModel.step(state, dt)` with the state in pinned host memory
copied in and out every step.  Under torchrun every rank runs its own replica
(the single-model path does not shard), so N ranks do N times the work.

`--impl reference` times the reference algorithm's CPU implementation (the
numpy/SuperLU oracle restatement) on the host cores, one bounded Newton-
iteration sample per step, in one process per core.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-Newton-its/s FI oil-water 1.1M cells: mixed-prec CPR vs FP64 GPU vs CPU"
UNIT = "cell*Newton-iterations/s"
WORKLOAD = dict(name="channelised oil-water 60x220x85 (1,122,000 cells), 10-day steps",
                dims=(60, 220, 85), cell_size=(6.1, 3.05, 0.61))
# Bounded CPU sample of the same model family: the channelised generator at
# 18 x 66 x 25 cells (29,700 cells, the full model's aspect ratios), first
# Newton iterations of the first timestep, SuperLU direct solve as the
# reference's default linear solver.  A smaller sample favours the CPU
# (direct-solve cost grows faster than linearly).
CPU_SAMPLE = dict(dims=(18, 66, 25), cell_size=(6.1 * 60 / 18, 3.05 * 220 / 66, 0.61 * 85 / 25))
# DRAM bytes per swept cell of one line_pcr_ell_kernel launch, from ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) on the 60x220x60 model
# (396,000 cells per colour).  The mixed-precision kernel has read and
# written its line-ordered r and z in FP32 since that capture, so its entry
# is left out (reported as null) until it is captured again.
PCR_DRAM_BYTES_PER_CELL = {"fp64": (119810560 + 4159744) / 396000.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="channelised", choices=["channelised", "ensemble", "blackoil", "transport"],
                    help="channelised: the headline benchmark; ensemble: config 3 on its own line; blackoil / "
                         "transport: those measurements of the other configurations on their own line "
                         "(--dims sets the grid)")
    ap.add_argument("--members", type=int, default=256, help="ensemble members (--workload ensemble)")
    ap.add_argument("--ens-graph", type=int, default=1, help="ensemble: replay each member's preconditioner as a graph")
    ap.add_argument("--ens-workers", type=int, default=0,
                    help="ensemble: host threads (0: the autotuned count, cached per SM count and ensemble shape)")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                    help="mixed: FP32 AMG and smoother blocks inside the FP64 FGMRES (the benchmark's method); fp64: all FP64")
    ap.add_argument("--dims", default=None, help="override grid dims, e.g. 30,110,40")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison arm")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the measurements of the other benchmark configurations")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--skip-implicit", action="store_true", help="transport workload: explicit transport only")
    ap.add_argument("--cpr", default="", help="CPR option overrides, e.g. amg_cycle=2,local_sweeps=1")
    ap.add_argument("--probe", type=int, default=0,
                    help="profiling probe: run this many Newton iterations of the first step and exit")
    ap.add_argument("--max-newton", type=int, default=60,
                    help="Newton iterations per step before a timestep cut; the reference's default is 25, "
                         "which the 10-day steps of this channelised model exceed (29-41 iterations)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# CPU oracle samples
# ---------------------------------------------------------------------------

def cpu_sample_worker(budget: float, seed: int = 2):
    """Newton iterations of the reference algorithm (oracle) on the CPU
    sample, until `budget` seconds are used; returns (cells, its, seconds)."""
    import scipy.sparse.linalg as spla
    from oracle import ow as oow
    from pymrst_b200 import cases
    case = cases.channelised(dims=CPU_SAMPLE["dims"], cell_size=CPU_SAMPLE["cell_size"], seed=seed,
                             n_smooth=int(round(CPU_SAMPLE["dims"][2] * 35 / 85)))
    prob = oow.build_problem(case.grid, case.rock, case.fluid.params, case.wells, gravity=case.gravity)
    st0 = oow.initial_state(prob, case.p0, case.sw0)
    st = st0.copy()
    cdp = oow.compute_cdp(prob, st0)
    its = 0
    t0 = time.perf_counter()
    while True:
        res, J = oow.assemble(prob, st0, st, case.dt, cdp)
        oow.converged(prob, res, case.dt, st)
        upd = spla.spsolve(J.tocsc(), -res)
        oow.apply_update(prob, st, upd)
        its += 1
        el = time.perf_counter() - t0
        if el >= budget or its >= 25:
            return prob.nc, its, el


def _pool_worker(args):
    budget, seed = args
    return cpu_sample_worker(budget, seed)


def run_reference(args):
    """The reference arm: the CPU algorithm on all host cores (one process
    per core, each a bounded sample), rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    budget = max(2.0, args.cpu_budget / 2)
    ctx = mp.get_context("spawn")
    values = []
    with ctx.Pool(cores) as pool:
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            out = pool.map(_pool_worker, [(budget, 2 + j) for j in range(cores)])
            wall = time.perf_counter() - t0
            v = sum(nc * its for nc, its, _ in out) / wall
            if i >= args.warmup:
                values.append((v, wall))
    v = float(np.mean([a for a, _ in values]))
    ms = float(np.mean([b for _, b in values])) * 1e3
    sample = (f"reference algorithm (numpy/SuperLU restatement) on the channelised generator at "
              f"{'x'.join(map(str, CPU_SAMPLE['dims']))} cells, Newton iterations of the first "
              f"10-day step for ~{budget:.0f} s per process, {cores} processes")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD["name"] + " (CPU runs a bounded sample)",
                       "sample_cells": int(np.prod(CPU_SAMPLE["dims"]))},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        def run():
            q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits"], capture_output=True,
                                         text=True, timeout=5).stdout.strip()
                    if out:
                        self.rows.append([s.strip() for s in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 3 + i and r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def kernel_roofline(model, x, x0, dt, torch, N, reps=20):
    """Live per-launch timing of the assembly and operator kernels on the
    current state, with their algorithmic bytes."""
    nc, nw = model.nc, model.nw
    nnzb = model.sizes["nnzb"]
    nf = model.N.shape[0]
    nvec = model.sizes["nvec"]
    cdp = torch.as_tensor(np.concatenate([np.zeros(np.asarray(w.cells).size) for w in model.wells]),
                          device="cuda")
    res, jac, well = model.assemble_device(x, x0, dt, cdp, True)
    y = torch.empty_like(x)
    stream = torch.cuda.current_stream()
    out = {}

    def time_it(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps * 1e-3

    # assembly: state (16 B) + previous state (16 B) + pv (8) + residual (16)
    # per cell; T, gdz (16 B) per interface; row_ptr/col/face code/diag_pos
    # indices (4 B each); the Jacobian blocks written (32 B each).
    asm_bytes = nc * (16 + 16 + 8 + 16 + 4 + 4) + nf * 16 + nnzb * (32 + 4 + 4)
    t = time_it(lambda: N.check(N.lib().pmb_ow_assemble(model._handle, N.ptr(x), N.ptr(x0), float(dt),
                                                         N.ptr(cdp), N.ptr(res), N.ptr(jac), N.ptr(well), 1)))
    out["assemble"] = dict(seconds=t, bytes=asm_bytes)
    # operator application: blocks (32 B) + column index (4 B) per block,
    # row_ptr, x read once, y written once
    spmv_bytes = nnzb * 36 + (nc + 1) * 4 + nvec * 16
    t = time_it(lambda: N.check(N.lib().pmb_ow_spmv(model._handle, N.ptr(jac), N.ptr(well), N.ptr(x), N.ptr(y))))
    out["spmv"] = dict(seconds=t, bytes=spmv_bytes)
    # CPR stages on this Jacobian, timed inside the library on its stream.
    s = model.solver_handle()
    N.check(N.lib().pmb_cpr_setup(s, N.ptr(jac), N.ptr(well), N.ptr(x)))
    z = torch.zeros_like(x)
    ms = N.C.c_double()
    sweeps = max(1, int(model.cpr_options.get("local_sweeps", 2)))
    N.check(N.lib().pmb_cpr_time_stage(s, 0, N.ptr(res), N.ptr(z), reps, N.C.byref(ms)))
    # one line Gauss-Seidel sweep (two colour launches of line_pcr_ell_kernel
    # and the well update) on the line-ordered operator copy: every block (FP64
    # 32 B or FP32 16 B) once, the column index of every block off the line
    # (4 B; the diagonal and the two line couplings need none), and per cell r
    # and z read and z written (FP64 16 B each, FP32 8 B in mixed precision)
    # and its perforation index (4 B).  The zero padding of short rows is not
    # counted.
    mixed = int(model.cpr_options.get("precision", 0)) == 1
    blk = 16 if mixed else 32
    lv = 8 if mixed else 16
    sweep_bytes = nnzb * blk + max(nnzb - 3 * nc, 0) * 4 + nc * (3 * lv + 4)
    out["line_gs_sweep"] = dict(seconds=ms.value * 1e-3 / sweeps, bytes=sweep_bytes)
    cb = (N.C.c_double * 8)()
    N.check(N.lib().pmb_cpr_bytes(s, cb))
    out["cpr_bytes"] = [float(v) for v in cb]
    # one visit of each level (the cycle from that level down), replayed from
    # a CUDA graph as the solver replays the preconditioner; level 0's visit
    # is one whole AMG cycle
    sizes = (N.C.c_int64 * 32)()
    nl = N.C.c_int32()
    N.check(N.lib().pmb_cpr_levels(s, 32, sizes, N.C.byref(nl)))
    levels = []
    nnz = N.C.c_int64()
    for lev in range(0, min(nl.value, 32)):
        N.check(N.lib().pmb_cpr_time_level(s, lev, 50, N.C.byref(ms), N.C.byref(nnz)))
        levels.append(dict(level=lev, rows=int(sizes[lev]), nnz=int(nnz.value), visit_ms=ms.value))
    out["amg_levels"] = levels
    out["amg_cycle"] = dict(seconds=levels[0]["visit_ms"] * 1e-3, bytes=float(cb[0]))
    # the whole preconditioner (restriction, AMG cycle, prolongation, the line
    # sweeps), replayed from its graph
    N.check(N.lib().pmb_cpr_time_stage(s, 3, N.ptr(res), N.ptr(z), reps, N.C.byref(ms)))
    out["preconditioner"] = dict(seconds=ms.value * 1e-3, bytes=float(cb[0] + sweeps * cb[1] + cb[3]))
    # set-up cost on this Jacobian: a fresh CPR handle (the host aggregation
    # of the pressure matrix, then the device Galerkin products, block
    # inverses and smoother bounds), then a refresh with the aggregates kept
    # (what every Newton iteration of the run pays); wall clock around device
    # synchronisations, since the first includes host work
    from pymrst_b200.ow_model import _opts_struct
    opts = _opts_struct(model.cpr_options)
    h2 = N.c_vp()
    N.check(N.lib().pmb_cpr_create(model._handle, N.C.byref(opts), N.C.byref(h2)))
    try:
        walls = []
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            N.check(N.lib().pmb_cpr_setup(h2, N.ptr(jac), N.ptr(well), N.ptr(x)))
            torch.cuda.synchronize()
            walls.append(time.perf_counter() - t0)
    finally:
        N.lib().pmb_cpr_destroy(h2)
    out["cpr_setup"] = dict(first_s=walls[0], refresh_s=walls[1])
    return out


# ---------------------------------------------------------------------------
# The other benchmark configurations, measured beside the headline one
# ---------------------------------------------------------------------------

def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def measure_incomp(torch, reps=5):
    """Config 0: incomp_tpfa on the 64x64x8 (32,768-cell) quarter five-spot,
    gravity off.  GPU: the public call (host arrays in and out, device
    assembly, PCG-AMG solve and reconstruction) and the device part alone,
    both CUDA-event timed after a warm-up call; CPU: the oracle's numpy
    assembly with SuperLU (the reference's algorithm), one run."""
    from oracle import incomp as oinc
    from pymrst_b200 import cases
    from pymrst_b200.incomp import _system, incomp_tpfa, init_single_fluid, init_state
    from pymrst_b200.ow_model import face_transmissibility_device
    c = cases.incompressible_quarter_five_spot()
    ht = face_transmissibility_device(c.grid, c.rock)[1]
    fluid = init_single_fluid(c.mu, c.rho)
    st0 = init_state(c.grid, c.wells, 0.0)
    run = lambda: incomp_tpfa(st0, c.grid, ht, fluid, wells=c.wells, rtol=1e-12, maxiter=1000)
    st = run()
    torch.cuda.synchronize()
    e0, e1 = _events(torch)
    e0.record()
    for _ in range(reps):
        st = run()
    e1.record()
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1) / reps
    syst = _system(c.grid, c.wells, False)
    mob = np.full((c.grid.cells.num, 1), 1.0 / c.mu)

    def device_part():
        syst.solve_device(1e-12, 1000)
        syst.reconstruct()

    device_part()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        device_part()
    e1.record()
    torch.cuda.synchronize()
    ms_dev = e0.elapsed_time(e1) / reps
    t0 = time.perf_counter()
    p_ref, bhp_ref, fp_ref, flux_ref, _ = oinc.incomp_tpfa(c.grid, ht, mob, [c.rho], None, None, None, c.wells)
    ms_cpu = (time.perf_counter() - t0) * 1e3
    return {"workload": "incompressible TPFA, 64x64x8 (32,768 cells), rate injector + bhp producer",
            "gpu_ms_per_call_e2e": ms_e2e, "gpu_ms_solve_and_reconstruct": ms_dev,
            "pcg_iterations": syst.last_iterations, "cpu_ms": ms_cpu,
            "cpu": "oracle restatement of incomp_tpfa (numpy assembly, SuperLU), one core",
            "speedup_e2e": ms_cpu / ms_e2e,
            "max_rel_pressure_vs_cpu": float(np.abs(st.pressure - p_ref).max() / np.abs(p_ref).max()),
            "max_rel_flux_vs_cpu": float(np.abs(st.flux - flux_ref).max() / np.abs(flux_ref).max())}


def measure_ow_fp64(torch, N, GpuOilWaterModel, run_report_step, cpu_budget=20.0):
    """Config 1: the FP64 oil-water five-spot on 100x100x10 cells, 20 steps of
    10 days from the initial state, all FP64 (library-default CPR); the
    whole schedule CUDA-event timed after a one-step warm-up on a copy.  CPU:
    Newton iterations of its first step by the oracle with SuperLU, at full
    size (one iteration, about 25 s on one core)."""
    import scipy.sparse.linalg as spla
    from oracle import ow as oow
    from pymrst_b200 import cases
    case = cases.five_spot(dims=(100, 100, 10), seed=1)
    model = GpuOilWaterModel(case.grid, case.rock, case.fluid, case.wells, gravity=case.gravity,
                             cpr_options=dict(precision=0))
    x = model.to_device(model.initial_state(case.p0, case.sw0))
    warm = x.clone()
    model.step_device(warm, case.dt)
    model.reset_cdp()
    saved = x.clone()

    def attempt(h):
        saved.copy_(x)
        ok, nit, _ = model.step_device(x, h)
        if not ok:
            x.copy_(saved)
        return ok, nit

    torch.cuda.synchronize()
    e0, e1 = _events(torch)
    its = 0
    e0.record()
    for _ in range(case.nsteps):
        its += run_report_step(attempt, case.dt, max_cuts=6)[0]
    e1.record()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) * 1e-3
    prob = oow.build_problem(case.grid, case.rock, case.fluid.params, case.wells, gravity=case.gravity)
    st0 = oow.initial_state(prob, case.p0, case.sw0)
    st = st0.copy()
    cdp = oow.compute_cdp(prob, st0)
    t0 = time.perf_counter()
    cits = 0
    while True:
        res, J = oow.assemble(prob, st0, st, case.dt, cdp)
        oow.apply_update(prob, st, spla.spsolve(J.tocsc(), -res))
        cits += 1
        if time.perf_counter() - t0 >= cpu_budget or cits >= 25:
            break
    csec = time.perf_counter() - t0
    gpu_v = model.nc * its / sec
    cpu_v = prob.nc * cits / csec
    return {"workload": "oil-water five-spot 100x100x10 (100,000 cells), 20 x 10 days, FP64",
            "value": gpu_v, "unit": UNIT, "ms_per_step": sec / case.nsteps * 1e3, "newton_iterations": its,
            "cpu_value": cpu_v, "cpu": f"oracle (numpy assembly, SuperLU) on the full model: {cits} Newton "
                                       f"iteration(s) of the first step in {csec:.1f} s, one core",
            "speedup": gpu_v / cpu_v}


def measure_adjoint(torch, GpuOilWaterModel, cpu_steps=3):
    """Config 4: the adjoint gradient of cumulative produced oil on the
    64x64x4 (16,384-cell) five-spot over 30 steps of 10 days, with respect
    to every well control of every step and every cell's log-permeability.
    GPU: one forward simulation alone, then the whole gradient (forward with
    checkpoints, recomputed segments, transposed solves), both CUDA-event
    timed after a 3-step warm-up; CPU: the oracle's forward and adjoint
    (SuperLU, the reference's algorithm) on the first `cpu_steps` steps."""
    from oracle import adjoint as oadj
    from oracle import ow as oow
    from pymrst_b200 import cases
    from pymrst_b200.adjoint import compute_gradient_adjoint, npv_objective
    c = cases.five_spot(dims=(64, 64, 4), seed=4, nsteps=30)
    m = GpuOilWaterModel(c.grid, c.rock, c.fluid, c.wells, gravity=c.gravity,
                         cpr_options=dict(amg_rebuild_interval=1_000_000))
    st0 = m.initial_state(c.p0, c.sw0)
    dts = np.full(c.nsteps, c.dt)
    u = np.tile([float(np.ravel(w.val)[0]) for w in c.wells], (c.nsteps, 1))
    obj = npv_objective(oil_price=1.0, water_cost=0.0, water_inj_cost=0.0)
    compute_gradient_adjoint(m, st0, dts[:3], u[:3], obj, perm_gradient=True)
    m.reset_cdp()
    x = m.to_device(st0)
    torch.cuda.synchronize()
    e0, e1 = _events(torch)
    e0.record()
    its = 0
    for n in range(c.nsteps):
        m.set_controls(u[n])
        ok, nit, _ = m.step_device(x, c.dt)
        its += nit
        if not ok:
            raise RuntimeError("forward step failed")
    e1.record()
    torch.cuda.synchronize()
    t_fwd = e0.elapsed_time(e1) * 1e-3
    m.reset_cdp()
    e0.record()
    res = compute_gradient_adjoint(m, st0, dts, u, obj, perm_gradient=True)
    e1.record()
    torch.cuda.synchronize()
    t_adj = e0.elapsed_time(e1) * 1e-3
    prob = oow.build_problem(c.grid, c.rock, c.fluid.params, c.wells, gravity=c.gravity)
    t0 = time.perf_counter()
    oadj.compute_gradient_adjoint(prob, oow.initial_state(prob, c.p0, c.sw0), dts[:cpu_steps], u[:cpu_steps])
    t_cpu = time.perf_counter() - t0
    return {"workload": "adjoint gradient, oil-water five-spot 64x64x4 (16,384 cells), 30 x 10 days, "
                        "d(cumulative oil)/d(controls, log k)",
            "gpu_forward_s": t_fwd, "gpu_gradient_s": t_adj, "gradient_over_forward": t_adj / t_fwd,
            "forward_newton_iterations": its, "checkpoint_every": res.stats["checkpoint_every"],
            "recomputed_steps": res.stats["recomputed_steps"],
            "transposed_krylov_iterations": res.stats["krylov_iterations"],
            "cpu_s_per_step": t_cpu / cpu_steps, "gpu_s_per_step": t_adj / c.nsteps,
            "speedup_per_step": (t_cpu / cpu_steps) / (t_adj / c.nsteps),
            "cpu": f"oracle forward + adjoint (numpy, SuperLU) over the first {cpu_steps} steps, one core"}


def measure_blackoil(torch, dims=(100, 100, 10), cpu_dims=(20, 20, 5), cpu_budget=30.0, cpu=True,
                     cpr_options=None):
    """The three-phase black-oil model with dissolved gas (the seeded
    lattice case of cases.blackoil_box: gas injectors, bhp producers, one
    oil-rate producer) over its seven steps (0.5 to 20 days), the whole
    schedule CUDA-event timed after a warm-up run on a copy of the state.
    CPU: the reference's own ThreePhaseBlackOilModelAD (its installed
    package, SuperLU) on the same generator at cpu_dims, steps until the
    budget is spent, one core."""
    from pymrst_b200 import cases
    from pymrst_b200.blackoil import GpuBlackOilModel
    case = cases.blackoil_box(dims=dims)
    model = GpuBlackOilModel(case.grid, case.rock, case.deck, case.wells, cpr_options=cpr_options)
    x0 = model.to_device(case.state)
    warm = x0.clone()
    for dt in case.dts[:2]:
        model.step_device(warm, float(dt))
    x = x0.clone()
    torch.cuda.synchronize()
    e0, e1 = _events(torch)
    its, krylov, failed = 0, 0, 0
    e0.record()
    for dt in case.dts:
        ok, nit, st = model.step_device(x, float(dt))
        its += nit
        krylov += int(st[2])
        failed += 0 if ok else 1
    e1.record()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) * 1e-3
    out = {"workload": f"black-oil (live oil, dry gas, switching) {dims[0]}x{dims[1]}x{dims[2]} "
                       f"({model.nc:,} cells, {model.nw} wells), steps of 0.5 to 20 days, FP64",
           "value": model.nc * its / sec, "unit": UNIT, "ms_per_step": sec / len(case.dts) * 1e3,
           "newton_iterations": its, "krylov_iterations": krylov, "failed_steps": failed,
           "saturated_cells_at_end": int((model.from_device(x).status == 3).sum())}
    ref = Path(__file__).resolve().parent / "baseline" / "_ref"
    if not cpu:
        return out
    if not (ref / "pymrst").is_dir():
        out["cpu"] = "the reference package is not installed under baseline/_ref"
        return out
    sys.path.insert(0, str(ref))
    from pymrst.gridprocessing import cart_grid, compute_geometry
    from pymrst.modules.ad_blackoil.models.three_phase_black_oil_model import BOState, ThreePhaseBlackOilModelAD
    from pymrst.modules.ad_props.props.init_deck_adi_fluid import init_deck_blackoil_fluid
    from pymrst.params import add_well, make_rock
    small = cases.blackoil_box(dims=cpu_dims)
    g = compute_geometry(cart_grid(list(cpu_dims), [d * 30.0 if i < 2 else d * 10.0 for i, d in enumerate(cpu_dims)]))
    rock = make_rock(g, np.asarray(small.rock.perm)[:, :1], 0.3)
    wells = None
    for w in small.wells:
        wells = add_well(wells, g, rock, w.cells, well_type=w.type, val=w.val, radius=0.1, compi=w.compi)
    rmodel = ThreePhaseBlackOilModelAD(g, rock, init_deck_blackoil_fluid(small.deck), wells)
    s0 = small.state
    st = BOState(pressure=s0.pressure.copy(), s=s0.s.copy(), rs=s0.rs.copy(), status=s0.status.copy(),
                 qWs=s0.qWs.copy(), qOs=s0.qOs.copy(), qGs=s0.qGs.copy(), bhp=s0.bhp.copy())
    t0 = time.perf_counter()
    cits, nsteps = 0, 0
    for dt in small.dts:
        st, ok, it = rmodel.step(st, float(dt))
        cits += it
        nsteps += 1
        if time.perf_counter() - t0 >= cpu_budget:
            break
    csec = time.perf_counter() - t0
    out.update(cpu_value=g.cells.num * cits / csec,
               cpu=f"the reference's ThreePhaseBlackOilModelAD (installed package, SuperLU) on the same generator "
                   f"at {cpu_dims[0]}x{cpu_dims[1]}x{cpu_dims[2]} ({g.cells.num} cells): {nsteps} step(s), {cits} "
                   f"Newton iterations in {csec:.1f} s, one core")
    out["speedup"] = out["value"] / out["cpu_value"]
    return out


def measure_transport(torch, n=256, cpu=True, implicit=True):
    """Sequential incompressible transport on an n x n quarter five-spot
    (rate injector and producer at opposite corners, the phase-3 Corey fluid,
    the permeability pattern of validate_phase3's qfs case): one device
    pressure solve, then implicit transport over 100 days and explicit
    transport with the stable-step estimate over 2 days, each CUDA-event
    timed after a warm-up call.  CPU: the oracle (numpy, SuperLU) on the same
    flux, implicit and explicit, bounded by the budget, one core."""
    from oracle import transport as otr
    from pymrst_b200.grid import cartesian_grid
    from pymrst_b200.incomp import State, incomp_tpfa
    from pymrst_b200.ow_model import face_transmissibility_device
    from pymrst_b200.params import CENTI, DARCY, DAY, MILLI, POISE, add_source, make_rock, pore_volume
    from pymrst_b200.transport import explicit_transport, implicit_transport, init_simple_fluid, transport_source
    g = cartesian_grid([n, n, 1], [500.0 * n / 32, 500.0 * n / 32, 10.0])
    nc = g.cells.num
    rock = make_rock(g, ((10 + (7 * np.arange(nc)) % 100) * MILLI * DARCY)[:, None], 0.2)
    fluid = init_simple_fluid(mu=np.array([1.0, 10.0]) * CENTI * POISE, rho=[1000.0, 700.0], n=[2.0, 2.0])
    rate = 5e-3 * (n / 32) ** 2
    src = add_source(add_source(None, [0], rate, sat=[[1.0, 0.0]]), [nc - 1], -rate, sat=[[0.0, 1.0]])
    new = lambda: State(pressure=np.zeros(nc), flux=np.zeros(g.faces.num),
                        s=np.column_stack([np.zeros(nc), np.ones(nc)]))
    st = incomp_tpfa(new(), g, face_transmissibility_device(g, rock)[1], fluid, src=src)
    flux = st.flux.copy()

    def run(kind, tf):
        s = new()
        s.flux = flux.copy()
        e0, e1 = _events(torch)
        torch.cuda.synchronize()
        e0.record()
        if kind == "implicit":
            implicit_transport(s, g, tf, rock, fluid, src=src)
        else:
            explicit_transport(s, g, tf, rock, fluid, src=src)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3, s.s[:, 0]

    t_imp, s_imp, stats = float("nan"), None, {}
    if implicit:
        run("implicit", 100 * DAY)
        t_imp, s_imp = run("implicit", 100 * DAY)
        stats = dict(implicit_transport.last_stats)
    run("explicit", 2 * DAY)
    t_exp, s_exp = run("explicit", 2 * DAY)
    nsub_gpu = explicit_transport.last_stats["substeps"]
    out = {"workload": f"incompressible transport, quarter five-spot {n}x{n} ({nc:,} cells), Corey n = 2, "
                       f"mu 1 / 10 cP",
           "implicit_100_days": {"gpu_s": t_imp, **stats},
           "explicit_2_days": {"gpu_s": t_exp, "substeps": nsub_gpu, "cell_substeps_per_s": nc * nsub_gpu / t_exp}}
    if not cpu or not implicit:
        return out
    # the oracle on the same flux
    Nall = np.asarray(g.faces.neighbors)
    internal = np.all(Nall >= 0, axis=1)
    q = transport_source(st, g, fluid, src=src)
    prob = otr.Problem(otr.Corey(fluid.mu, fluid.rho, fluid.n), Nall[internal], flux[internal],
                       np.zeros(int(internal.sum())), q, pore_volume(g, rock))
    t0 = time.perf_counter()
    s_cpu, nsub = prob.explicit(np.zeros(nc), 2 * DAY, np.zeros(int(internal.sum())))
    t_cpu_exp = time.perf_counter() - t0
    t0 = time.perf_counter()
    s_cpu_imp = prob.implicit(np.zeros(nc), 100 * DAY)
    t_cpu_imp = time.perf_counter() - t0
    return {"workload": f"incompressible transport, quarter five-spot {n}x{n} ({nc:,} cells), Corey n = 2, "
                        f"mu 1 / 10 cP",
            "implicit_100_days": {"gpu_s": t_imp, "cpu_s": t_cpu_imp, "speedup": t_cpu_imp / t_imp,
                                  "max_abs_ds_vs_cpu": float(np.abs(s_imp - s_cpu_imp).max()), **stats},
            "explicit_2_days": {"gpu_s": t_exp, "cpu_s": t_cpu_exp, "speedup": t_cpu_exp / t_exp, "substeps": nsub_gpu,
                                 "cpu_substeps": nsub, "cell_substeps_per_s": nc * nsub_gpu / t_exp,
                                 "max_abs_ds_vs_cpu": float(np.abs(s_exp - s_cpu).max())},
            "cpu": "oracle (numpy; SuperLU for the implicit systems) on the same flux, one core"}


def cpr_overrides(text: str) -> dict:
    """`--cpr k=v,...` as CPR options."""
    out = {}
    for kv in filter(None, text.split(",")):
        k, v = kv.split("=")
        out[k] = float(v) if k in ("rtol", "amg_theta", "inner_rtol") else int(v)
    return out


def run_side_workload(args):
    """One of the other configurations' measurements as its own JSON line
    (rank 0, one GPU)."""
    import torch
    dims = tuple(int(v) for v in args.dims.split(",")) if args.dims else None
    if args.workload == "blackoil":
        out = measure_blackoil(torch, dims=dims or (100, 100, 10), cpu=not args.no_cpu_baseline,
                               cpr_options=cpr_overrides(args.cpr) or None)
    else:
        out = measure_transport(torch, n=dims[0] if dims else 256, cpu=not args.no_cpu_baseline,
                                implicit=not args.skip_implicit)
    print(json.dumps({"workload": args.workload, **out}), flush=True)


def run_ensemble_workload(args):
    """Config 3 (`--workload ensemble`): the seeded realisations (nx, ny in
    16..64, nz in 2..8, an independent lognormal permeability and a five-spot
    each) over `--steps` report steps of 30 days.  GPU: every member on its
    own model, host threads with a stream each (their count autotuned on the
    first report step of 64 members and cached; each member's results are
    those of its single run), wall time bracketed by device synchronisations
    (the work is spread over many streams); CPU: the oracle (numpy + SuperLU;
    the reference's run_ensemble runs members one after another) on the first
    member's first Newton iterations, per cell and iteration."""
    import scipy.sparse.linalg as spla
    import torch
    from oracle import ow as oow
    from pymrst_b200 import cases
    from pymrst_b200.build import build
    from pymrst_b200.ensemble import simulate_members_concurrently, tune_workers
    from pymrst_b200.ow_model import GpuOilWaterModel
    if int(os.environ.get("RANK", "0")) != 0:
        return
    build()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    reals = cases.ensemble_realisations(n=args.members, nsteps=args.steps)
    members = [(c.grid, c.rock, c.wells) for c in reals]
    st0 = [GpuOilWaterModel(c.grid, c.rock, c.fluid, c.wells, gravity=c.gravity).initial_state(c.p0, c.sw0)
           for c in reals]
    dts = np.full(args.steps, reals[0].dt)
    cells = np.array([c.grid.cells.num for c in reals])
    tuned = tune_workers(members, reals[0].fluid, st0, dts, gravity=reals[0].gravity,
                         replay_graph=bool(args.ens_graph))
    workers = args.ens_workers or tuned["workers"]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, its = simulate_members_concurrently(members, reals[0].fluid, st0, dts, gravity=reals[0].gravity,
                                           workers=workers, replay_graph=bool(args.ens_graph))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    work = float(np.sum(cells[:, None] * its))
    c = reals[0]
    prob = oow.build_problem(c.grid, c.rock, c.fluid.params, c.wells, gravity=c.gravity)
    s0 = oow.initial_state(prob, c.p0, c.sw0)
    st = s0.copy()
    cdp = oow.compute_cdp(prob, s0)
    t1 = time.perf_counter()
    cits = 0
    while time.perf_counter() - t1 < args.cpu_budget and cits < 25:
        res, J = oow.assemble(prob, s0, st, c.dt, cdp)
        oow.apply_update(prob, st, spla.spsolve(J.tocsc(), -res))
        cits += 1
    cpu = prob.nc * cits / (time.perf_counter() - t1)
    line = {"metric": "cell-Newton-its/s, oil-water ensemble (config 3)", "value": work / wall,
            "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": 1, "ms_per_step": wall / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded realisations)",
            "config": {"workload": f"{args.members} oil-water realisations, nx, ny in 16..64, nz in 2..8, "
                                   f"{args.steps} x 30 days", "cells": int(cells.sum()),
                       "newton_iterations": int(its.sum()),
                       "runner": f"one model per member, {workers} threads with a stream each, preconditioner "
                                 + ("replayed as a CUDA graph" if args.ens_graph else "launched kernel by kernel"),
                       "autotune": {"key": tuned["key"], "workers": tuned["workers"],
                                    "trial_seconds": {str(k): v for k, v in tuned["trials"].items()}},
                       "timing": "wall clock between device synchronisations"},
            "cpu_baseline": {"value": cpu, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": f"oracle (numpy, SuperLU) on member 0 ({prob.nc} cells): {cits} Newton "
                                       f"iterations of its first step"}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist
    from pymrst_b200 import _native as N
    from pymrst_b200 import cases
    from pymrst_b200.build import build
    from pymrst_b200.ow_model import GpuOilWaterModel
    from pymrst_b200.replicas import reduce_timing
    from pymrst_b200.schedule import run_report_step

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if rank == 0:
        build()
    if world > 1:
        dist.barrier()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # bounded CPU sample before any heavy GPU work (single process)
        nc_s, its_s, el = cpu_sample_worker(args.cpu_budget)
        cpu = {"value": nc_s * its_s / el, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": (f"reference algorithm (numpy/SuperLU restatement) on the channelised generator at "
                          f"{'x'.join(map(str, CPU_SAMPLE['dims']))} = {nc_s} cells: {its_s} Newton "
                          f"iterations of the first 10-day step in {el:.1f} s, one core")}

    dims = tuple(int(v) for v in args.dims.split(",")) if args.dims else WORKLOAD["dims"]
    n_smooth = int(round(dims[2] * 35 / 85))
    case = cases.channelised(dims=dims, cell_size=WORKLOAD["cell_size"], n_smooth=n_smooth)
    # CPR options tuned on this workload (reported in config.cpr): Chebyshev
    # degree 3 and 7 line sweeps need 26% fewer Krylov iterations here than
    # the library defaults (degree 2, 4 sweeps), which the batched ensemble
    # needs; degree 2 on the levels below the K-cycle, which every cycle
    # visits eight times; aggregates are built once per run
    copts = dict(rtol=1e-8, maxiter=400, restart=50, amg_rebuild_interval=1_000_000,
                 precision=1 if args.precision == "mixed" else 0, amg_cycle=3, local_sweeps=7,
                 amg_smoother_degree=3, amg_coarse_degree=2, amg_theta=0.1)
    copts.update(cpr_overrides(args.cpr))
    model = GpuOilWaterModel(case.grid, case.rock, case.fluid, case.wells, gravity=case.gravity,
                             cpr_options=copts, max_iterations=args.max_newton)
    stream = torch.cuda.current_stream()
    x = model.to_device(model.initial_state(case.p0, case.sw0))
    dt = case.dt
    if args.probe:
        model.max_iterations = args.probe
        torch.cuda.synchronize()
        ok, nit, st = model.step_device(x, dt)
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"probe": True, "cells": model.nc, "newton": nit, "krylov": int(st[2]),
                              "amg_levels": model.cpr_levels()}), flush=True)
        return

    def run_steps(mdl, xv, nsteps, snapshots=None, per_step=None):
        """Report steps of the schedule with the reference's halving cuts
        (schedule.run_report_step); returns (Newton its, Krylov its, cuts).
        With `snapshots`, a device copy of the state after each report step
        is kept (a device-to-device copy, about 10 us per step)."""
        tot = [0, 0, 0]
        saved = xv.clone()
        for _ in range(nsteps):
            kry = [0]

            def attempt(h):
                saved.copy_(xv)
                ok, nit, st = mdl.step_device(xv, h)
                kry[0] += int(st[2])
                if os.environ.get("PMB_VERBOSE") == "1":
                    print(f"# step dt={h / 86400:.3g} d ok={ok} newton={nit} krylov={int(st[2])} "
                          f"cnv={st[4]:.2e} mb={st[5]:.2e} {getattr(mdl, 'last_failure', '') if not ok else ''}",
                          file=sys.stderr, flush=True)
                if not ok:
                    xv.copy_(saved)
                return ok, nit

            its, cuts = run_report_step(attempt, dt, max_cuts=6)
            tot[0] += its
            tot[1] += kry[0]
            tot[2] += cuts
            if snapshots is not None:
                snapshots.append(xv.clone())
            if per_step is not None:
                per_step.append(its)
        return tot

    def one_step(xv):
        i, k, c = run_steps(model, xv, 1)
        return i, k, c

    x_before_last = None
    for i in range(args.warmup):
        if i == args.warmup - 1:
            x_before_last = x.clone()
        one_step(x)
    torch.cuda.synchronize()
    x_e2e_start = x.clone()
    l0 = N.launch_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    snaps, its_steps = [], []
    with ClockSampler(local) as clocks:
        e0.record(stream)
        its_total, kry_total, cuts_total = run_steps(model, x, args.steps, snaps, its_steps)
        e1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = N.launch_count() - l0
    if os.environ.get("PMB_PROFILE") == "1" and rank == 0:
        prof = N.profile_report(reset=True)
        total = e0.elapsed_time(e1)
        print(f"# timed region {total:.1f} ms; phases (total ms, count, ms each):", file=sys.stderr)
        for k, (ms, cnt) in sorted(prof.items(), key=lambda kv: -kv[1][0]):
            print(f"#   {k:28s} {ms:10.2f} {cnt:7d} {ms / max(cnt, 1):9.4f}", file=sys.stderr)
    sec, cell_its = reduce_timing(e0.elapsed_time(e1) * 1e-3, float(its_total) * model.nc)
    value = cell_its / sec

    # e2e: the same steps through the public host-state API (pinned copies in
    # and out each step)
    st_host = model.from_device(x_e2e_start)
    model.step(st_host, dt)  # warm the staging buffers
    st_host = model.from_device(x_e2e_start)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    its_e2e = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        # a report step through the public API, cuts as in the driver
        holder = [st_host]

        def attempt(h):
            new, ok, nit = model.step(holder[0], h)
            if ok:
                holder[0] = new
            return ok, nit

        nit, _ = run_report_step(attempt, dt, max_cuts=6)
        its_e2e += nit
        st_host = holder[0]
    torch.cuda.synchronize()
    sec_e2e, cell_its_e2e = reduce_timing(time.perf_counter() - t0, float(its_e2e) * model.nc)
    nvec_bytes = model.sizes["nvec"] * 8

    # The FP64 form of the same solve (every preconditioner array in FP64)
    # from the same start state, timed the same way, and the difference of
    # the mixed-precision states from it after every report step.
    fp64 = None
    if args.precision == "mixed" and not args.no_fp64:
        copts64 = dict(copts, precision=0)
        model64 = GpuOilWaterModel(case.grid, case.rock, case.fluid, case.wells, gravity=case.gravity,
                                   cpr_options=copts64, max_iterations=args.max_newton)
        # untimed: aggregation and graph capture on the last warm-up step, which
        # also leaves the model's previous-step well pressure drops where the
        # mixed run had them when its timed steps began
        x64 = (x_before_last if x_before_last is not None else x_e2e_start).clone()
        if x_before_last is not None:
            run_steps(model64, x64, 1)
        x64.copy_(x_e2e_start)
        snaps64, its64 = [], []
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        n64, k64, c64 = run_steps(model64, x64, args.steps, snaps64, its64)
        f1.record(stream)
        torch.cuda.synchronize()
        sec64, cell_its64 = reduce_timing(f0.elapsed_time(f1) * 1e-3, float(n64) * model.nc)
        nc2 = 2 * model.nc
        errs = []
        for a, b in zip(snaps, snaps64):
            pa, pb = a[0:nc2:2], b[0:nc2:2]
            errs.append((float((pa - pb).abs().max() / pb.abs().max()),
                         float((a[1:nc2:2] - b[1:nc2:2]).abs().max())))
        fp64 = {"value": cell_its64 / sec64, "ms_per_step": sec64 / args.steps * 1e3, "newton_iterations": n64,
                "krylov_iterations": k64, "cuts": c64, "speedup_mixed_over_fp64": value / (cell_its64 / sec64)}
        mixed_vs_fp64 = {"max_rel_pressure": max(e[0] for e in errs), "max_abs_sw": max(e[1] for e in errs),
                         "per_step_rel_pressure": [e[0] for e in errs], "per_step_abs_sw": [e[1] for e in errs],
                         "newton_per_step_mixed": its_steps, "newton_per_step_fp64": its64,
                         "equal_newton_counts": its_steps == its64}
        del model64, snaps64
    del snaps

    kr = kernel_roofline(model, x, x_e2e_start, dt, torch, N)
    configs = {}
    if not args.no_configs and rank == 0 and world == 1:
        for name, fn in (("incomp_64x64x8", lambda: measure_incomp(torch)),
                         ("ow_fp64_100x100x10", lambda: measure_ow_fp64(torch, N, GpuOilWaterModel, run_report_step,
                                                                        args.cpu_budget)),
                         ("adjoint_64x64x4", lambda: measure_adjoint(torch, GpuOilWaterModel)),
                         ("blackoil_100x100x10", lambda: measure_blackoil(torch)),
                         ("transport_256x256", lambda: measure_transport(torch))):
            try:
                configs[name] = fn()
            except Exception as e:  # a secondary measurement must not hide the headline line
                configs[name] = {"error": f"{type(e).__name__}: {e}"}
    peak, peak_kind = peaks()
    # whole-step algorithmic bytes from the recorded counts: per Newton
    # iteration the assembly, the convergence check and update, and one
    # preconditioner setup; per Krylov iteration the operator product, one
    # preconditioner application (AMG cycle, restriction and prolongation,
    # every second-stage sweep) and the Gram-Schmidt traffic at the mean
    # iteration count per solve
    cb = kr["cpr_bytes"]
    nvec = cb[5]
    m_it = kry_total / max(its_total, 1)
    orth = its_total * (m_it * (m_it - 1) + 6 * m_it) * nvec * 8
    sweeps = int(copts.get("local_sweeps", 1))
    per_newton = kr["assemble"]["bytes"] + cb[4] + cb[6] + model.nc * 40 + nvec * 24
    per_krylov = cb[2] + cb[0] + cb[3] + sweeps * cb[1]
    step_bytes = (its_total * per_newton + kry_total * per_krylov + orth) / args.steps
    step_ach = step_bytes / (sec / args.steps) / 1e9
    dom = kr["line_gs_sweep"]
    ach = dom["bytes"] / dom["seconds"] / 1e9
    # DRAM traffic of one line_pcr_ell_kernel launch (one colour, half the cells),
    # scaled from the ncu capture of dram__bytes_read.sum + dram__bytes_write.sum
    # on the 60x220x60 model (396,000 cells per colour)
    traffic = PCR_DRAM_BYTES_PER_CELL.get(args.precision)
    traffic = traffic * model.nc / 2 if traffic else None
    if world > 1:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic (seeded channelised permeability, five-spot wells)",
            "config": {"workload": WORKLOAD["name"], "cells": model.nc, "wells": model.nw,
                       "dt_days": dt / 86400.0, "precision": args.precision,
                       "max_newton_iterations": args.max_newton,
                       "newton_iterations": its_total, "krylov_iterations": kry_total, "cuts": cuts_total,
                       "cpr": {k: copts[k] for k in copts}, "amg_levels": model.cpr_levels(),
                       "l2": "inputs larger than L2 (Jacobian %.0f MB)" % (model.sizes['nnzb'] * 32 / 1e6),
                       "parallelism": f"{world} independent replicas" if world > 1 else "single GPU"},
            "e2e": {"value": cell_its_e2e / sec_e2e, "unit": UNIT, "h2d_bytes_per_step": nvec_bytes,
                    "d2h_bytes_per_step": nvec_bytes},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm",
                         "kernel": "line_pcr_ell_kernel (vertical-line block Gauss-Seidel, one colour per launch)",
                         "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes": dom["bytes"] / 2,
                         "step": {"bytes_per_step": step_bytes, "achieved": step_ach, "frac": step_ach / peak,
                                  "per_newton_bytes": per_newton, "per_krylov_bytes": per_krylov,
                                  "orthogonalisation_bytes_per_step": orth / args.steps},
                         "kernels": {k: {"ms": v["seconds"] * 1e3, "bytes": v["bytes"],
                                         "GBps": (v["bytes"] / v["seconds"] / 1e9) if v["bytes"] else None}
                                     for k, v in kr.items() if k not in ("cpr_bytes", "cpr_setup", "amg_levels")},
                         "amg_level_visits": kr["amg_levels"],
                         "cpr_setup_ms": {"first_with_host_aggregation": kr["cpr_setup"]["first_s"] * 1e3,
                                          "refresh": kr["cpr_setup"]["refresh_s"] * 1e3}},
            "clocks": clocks.summary(),
        }
        if configs:
            line["other_configs"] = configs
        if fp64 is not None:
            line["fp64"] = fp64
            line["mixed_vs_fp64"] = mixed_vs_fp64
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "ensemble":
        run_ensemble_workload(args)
    elif args.workload in ("blackoil", "transport"):
        run_side_workload(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
