"""Throughput benchmark of the euler_compare hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the configuration the headline metric is quoted on): explicit O2
HLLC, FP64, on the 2560x640 shock-density-bubble grid (domain [0,2]x[0,0.5],
reflecting bottom wall, post-shock inflow, outflow right/top; the reference's
own problem definition), initial state from its initializer.  One step = one
pass of the hot path over the grid: the fused kernel computes dt from the
previous step's CFL reduction, reconstructs (MUSCL, minmod), evaluates every
HLLC face flux, updates the state and reduces the next CFL rate and the
admissibility diagnostics.

value: cell-updates/s with the state resident in HBM (CUDA events around each
step's launch on the launching stream, through the C entry point without the
degenerate-count read-back; L2 flushed before every timed step by writing a
256 MiB buffer and reading it back, since the 52 MB state would otherwise stay
in the 126 MB L2; the read-back leaves clean lines, so the step does not pay
for writing back the flush buffer).
e2e: the same metric through the C ABI with HOST buffers: each step is one
ecg_euler_fv_one_step_host call that copies the step's input from pinned host
memory to the device, steps it and copies the result back, pipelined over row
bands so that both copy directions and the step overlap (dt from
compute_euler_dt of the input), as a drop-in for a host-resident MultiFab.

--impl reference: the reference's own CPU code (oracle/_ref: the reference
headers built with g++ against a single-box AMReX shim) on
the same workload, on this machine's host cores (rows split over all host
threads); one step = the driver's loop
body compute_euler_dt -> euler_fv_one_step -> compute_diagnostics.

Two more measurements ride on the same JSON line at N=1 (skip them with
--no-extra-legs): "imex", the second half of the metric (Gresho vortex at
M = 0.01 on 256^2 and on 768^2, and the 2560x640 bubble, IMEX T1/S2: ms per
step of the all-FP64 GMRES solve and of the FP32-basis / FP64-arithmetic
solve, their iterations, and the relative drift between the two states; its
mixed_speedup is the 256^2 Gresho case's), and "batched" (64 seeded Riemann
solves of uneven sizes advanced by one persistent launch per step for 200
steps).

Multi-GPU: the single 2560x640 solve does not shard without a halo exchange,
so N GPUs run N independent replicas (weak scaling); value is the sum over
ranks of cells / (max over ranks of the timed region).
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NY = 2560, 640
METRIC = "cell-updates/s at 2560x640 FP64 (%HBM); IMEX mixed vs FP64 time at equal L1"
UNIT = "cell-updates/s"
BYTES_PER_CELL = 64  # read 4 FP64 conserved values, write 4
WORKLOAD_KV = {
    "euler.problem": "shock_density_bubble_2d",
    "amr.n_cell": f"{NX} {NY}",
    "euler.method": "explicit",
    "euler.riemann": "hllc",
    "euler.spatial_order": 2,
    "euler.slope_limiter": "minmod",
    "euler.cfl": 0.45,
    "stop_time": 1.0,
}
CONFIG = {
    "workload": "shock_density_bubble_2d 2560x640, explicit O2 MUSCL-minmod HLLC, FP64, CFL 0.45",
    "grid": [NX, NY],
    "domain": [[0.0, 2.0], [0.0, 0.5]],
    "riemann": "hllc",
    "l2": "flushed before every timed step (256 MiB written, then read back)",
    "parallelism": "replicas",
}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def step_profile():
    """The committed ncu summary of the step kernel: DRAM bytes per launch and
    FP64 flops per cell (opcode counts of the same capture)."""
    p = os.path.join(ROOT, "profiles", "fv_march_hllc_bubble_2560x640.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return None
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def init_dist(world, backend):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist

    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def max_over_ranks(dist, x, device=None):
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, x, device=None):
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------------------------------------
# CPU legs (the oracle is a checker/baseline only)


def cpu_reference_step_rate(steps, threads=None, grid=(NX, NY)):
    """The reference's CPU code on the workload: cell-updates/s over `steps`
    driver-loop bodies on the full grid.  Returns (value, kind, cores, sample)."""
    from tests.oracle import REF_SO, Oracle, RefOracle

    if threads:
        os.environ["ECG_REF_THREADS"] = str(threads)
    kv = dict(WORKLOAD_KV, **{"amr.n_cell": f"{grid[0]} {grid[1]}"})
    if os.path.exists(REF_SO):
        r = RefOracle()
        r.configure(kv)
        u = r.initialize()
        t = 0.0
        dt = r.euler_dt(u, t)
        r.step(u, dt, t)  # warm
        t0 = time.perf_counter()
        for _ in range(steps):
            dt = r.euler_dt(u, t)
            u, _ = r.step(u, dt, t)
            r.diagnostics(u)
            t += dt
        el = time.perf_counter() - t0
        kind = "reference"
    else:
        from amrex_euler_allmach_explicit_imex_b200.config import read_config

        o = Oracle()
        cfg = read_config(kv).cfg
        u = o.initialize(cfg)
        t = 0.0
        t0 = time.perf_counter()
        for _ in range(steps):
            dt = o.euler_dt(cfg, u, t)
            u, _ = o.step(cfg, u, dt, t)
            o.diagnostics(cfg, u)
            t += dt
        el = time.perf_counter() - t0
        kind = "port"
    cores = int(os.environ.get("ECG_REF_THREADS", "1")) if kind == "reference" else 1
    value = grid[0] * grid[1] * steps / el
    sample = f"{steps} driver-loop steps (dt, euler_fv_one_step, diagnostics) on the full {grid[0]}x{grid[1]} grid"
    return value, kind, cores, sample


def run_reference_arm(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    steps = max(1, args.steps)
    from tests.oracle import REF_SO

    if not os.path.exists(REF_SO):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built on this machine"}))
        return 0
    os.environ["ECG_REF_THREADS"] = str(threads)
    # warmup
    cpu_reference_step_rate(max(1, min(args.warmup, 2)), threads)
    value, kind, cores, sample = cpu_reference_step_rate(steps, threads)
    ms = NX * NY / value * 1e3
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (the reference's own shock-density-bubble initializer)", "config": CONFIG,
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------------------------
# GPU arm


def imex_kv(n, mach):
    return {
        "amr.n_cell": f"{n} {n}", "geometry.is_periodic": "1 1", "euler.problem": "gresho_vortex",
        "euler.vortex_center": "0.5 0.5", "euler.mach": mach, "euler.pressure": 1.0 / (1.4 * mach * mach),
        "euler.method": "imex", "euler.spatial_order": 2, "euler.imex_acoustic_startup": 0,
        "euler.imex_picard_iterations": 4, "euler.imex_solver_tol": "1e-10", "euler.imex_solver_max_iter": 200,
        "euler.imex_cfl": 0.4, "stop_time": 1.0,
    }


def bubble_imex_kv(nx, ny):
    """The shock-density bubble's IMEX settings (imex_cfl 0.45, 4 Picard
    passes, GMRES tol 1e-10 / 200 iterations, no acoustic start-up or cap)."""
    return {
        "amr.n_cell": f"{nx} {ny}", "geometry.prob_hi": "2 0.5", "euler.problem": "shock_density_bubble_2d",
        "euler.method": "imex", "euler.spatial_order": 2, "euler.imex_acoustic_startup": 0,
        "euler.imex_acoustic_cfl_cap": 0, "euler.imex_picard_iterations": 4, "euler.imex_solver_tol": "1e-10",
        "euler.imex_solver_max_iter": 200, "euler.imex_cfl": 0.45, "stop_time": 1.0,
    }


# (name, configuration): the Gresho configuration of the metric, a grid whose
# Krylov basis no longer fits in L2 (the FP32 basis halves the bytes of the
# sweeps that dominate there; at 256^2 the solve is bound by barrier latency),
# and the bubble's IMEX step (a few GMRES iterations a solve)
def mach122_imex_kv(nx, ny):
    """The Mach 1.22 bubble on [0,4]x[0,1] with the bubble's IMEX settings."""
    kv = bubble_imex_kv(nx, ny)
    kv.update({"euler.problem": "shock_bubble_mach122", "geometry.prob_hi": "4 1"})
    return kv


IMEX_CASES = [("gresho_vortex 256x256 periodic, M=0.01", imex_kv(256, 0.01)),
              ("gresho_vortex 256x256 periodic, M=0.1", imex_kv(256, 0.1)),
              ("gresho_vortex 256x256 periodic, M=0.001", imex_kv(256, 0.001)),
              ("gresho_vortex 768x768 periodic, M=0.01", imex_kv(768, 0.01)),
              ("shock_density_bubble_2d 640x160", bubble_imex_kv(640, 160)),
              ("shock_density_bubble_2d 2560x640", bubble_imex_kv(2560, 640)),
              ("shock_bubble_mach122 2560x640 on [0,4]x[0,1]", mach122_imex_kv(2560, 640))]

# Algorithmic bytes of an IMEX step outside GMRES, per cell: the star update
# (read U, write U*, p, K: 88 B), per Picard pass the assembly (80 B: U*, p,
# K read, face enthalpies and rhs written) and the p / eq54 momentum refresh
# (56 B: x read, p written; m*, p read, K written), and the closeout (48 B).
# The GMRES sweeps' bytes come from the solve's own count of the vector
# sweeps it ran (ecg_imex_diag.gmres_vector_bytes).
IMEX_STAR_B, IMEX_PICARD_B, IMEX_CLOSE_B = 88, 80 + 56, 48


def imex_leg(dev, stream, steps=3, only_case=None):
    """Each IMEX_CASES configuration, IMEX T1/S2 (4 Picard solves, GMRES tol
    1e-10): time per step of the all-FP64 solve and of the FP32-basis /
    FP64-arithmetic solve on the same GPU, their GMRES iterations and solver
    statuses, the step's algorithmic bytes and HBM fraction, and the drift
    between the two states after `steps` + 1 steps (max-norm relative, and the
    relative difference of the density in L1)."""
    import torch

    from amrex_euler_allmach_explicit_imex_b200 import api
    from amrex_euler_allmach_explicit_imex_b200.config import read_config

    peak, _ = peaks()
    cases = []
    for ci, (name, kv) in enumerate(IMEX_CASES):
        if only_case is not None and ci != only_case:
            continue
        cfg = read_config(kv).cfg
        cells = cfg.n_cell[0] * cfg.n_cell[1]
        out = {}
        states = {}
        # "fp64_again": the FP64 run once more, whose only difference from the
        # first is the order of the GMRES kernel's atomic sums: its drift from
        # the first is how far two solves stopped at the 1e-10 tolerance lie
        # apart anyway, the floor for the mixed solve's drift
        for prec in ("fp64", "mixed", "fp64_again"):
            with api.Context(cfg, imex_precision="mixed" if prec == "mixed" else "fp64", device=dev.index or 0,
                             stream=stream.cuda_stream) as ctx:
                api.initialize_state(ctx)
                t = 0.0
                ms, its, statuses, gbytes, fp32 = [], [], [], [], []
                for k in range(steps + 1):
                    dt, _ = api.compute_imex_dt(ctx, t)
                    a = torch.cuda.Event(enable_timing=True)
                    b = torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    d = api.euler_imex_bdltv20_o1_source_map_picard_one_step(ctx, dt)
                    b.record(stream)
                    b.synchronize()
                    statuses.append(api.solver_status_str(d.solver_status))
                    if k > 0:
                        ms.append(a.elapsed_time(b))
                        its.append(d.gmres_inner_iterations if prec == "mixed" else d.solver_iterations)
                        gbytes.append(d.gmres_vector_bytes)
                        fp32.append(d.gmres_fp32_basis)
                    t += dt
                states[prec] = ctx.download()
                if prec == "fp64_again":
                    continue
                med = statistics.median(ms)
                gb = statistics.median(gbytes)
                other = cells * (IMEX_STAR_B + cfg.imex_picard_iterations * IMEX_PICARD_B + IMEX_CLOSE_B)
                step_bytes = gb + other
                out[prec] = {"ms_per_step": med, "gmres_iterations": its, "status": statuses[-1],
                             "fp32_basis_steps": sum(fp32),
                             "step_statuses": statuses, "gmres_bytes_per_step": gb, "step_bytes": step_bytes,
                             "achieved_gbs": step_bytes / (med * 1e-3) / 1e9,
                             "hbm_frac": step_bytes / (med * 1e-3) / 1e9 / peak}
        f, m, f2 = states["fp64"], states["mixed"], states["fp64_again"]
        drift = float(np.abs(f - m).max() / np.abs(f).max())
        l1drift = float(np.abs(f[0] - m[0]).sum() / np.abs(f[0]).sum())
        floor = float(np.abs(f - f2).max() / np.abs(f).max())
        l1floor = float(np.abs(f[0] - f2[0]).sum() / np.abs(f[0]).sum())
        ok = all(x.startswith("converged") for p in ("fp64", "mixed") for x in out[p]["step_statuses"])
        cases.append({"workload": name + ", IMEX T1/S2, 4 Picard, GMRES tol 1e-10", "fp64": out["fp64"],
                      "mixed": out["mixed"], "mixed_speedup": out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"],
                      "state_rel_drift": drift, "density_l1_rel_drift": l1drift,
                      "fp64_repeat_state_rel_drift": floor, "fp64_repeat_density_l1_rel_drift": l1floor,
                      "all_steps_converged": ok})
    return {"steps_timed": steps, "mixed_speedup": cases[0]["mixed_speedup"],
            "bytes_model": "GMRES: the solve's count of vector sweeps (8 B per FP64 entry, 4 per FP32 basis entry); "
                           "outside GMRES: 88 B/cell star + 136 B/cell per Picard pass + 48 B/cell closeout",
            "cases": cases}


def hllcp_leg(dev, stream, steps=20):
    """The explicit step with the low-Mach-corrected HLLC-P flux
    (xie_am_hllc_p, 5-face pressure sensor): the Gresho vortex at 256^2,
    M = 0.01 (CFL 0.5), and the shock-density bubble at 2560x640 (CFL 0.45);
    CUDA events around each step, L2 flushed before each."""
    import torch

    from amrex_euler_allmach_explicit_imex_b200 import _lib, api
    from amrex_euler_allmach_explicit_imex_b200.config import read_config

    lib = _lib.load()
    peak, _ = peaks()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    sink = torch.empty((), dtype=torch.float32, device=dev)
    cases = [("gresho_vortex 256x256 periodic, M=0.01, xie_am_hllc_p, CFL 0.5",
              dict(imex_kv(256, 0.01), **{"euler.method": "explicit", "euler.riemann": "xie_am_hllc_p",
                                          "euler.cfl": 0.5})),
             ("shock_density_bubble_2d 2560x640, xie_am_hllc_p, CFL 0.45",
              dict(WORKLOAD_KV, **{"euler.riemann": "xie_am_hllc_p"}))]
    res = []
    for name, kv in cases:
        cfg = read_config(kv).cfg
        cells = cfg.n_cell[0] * cfg.n_cell[1]
        with api.Context(cfg, arith="fast", device=dev.index or 0, stream=stream.cuda_stream) as ctx:
            api.initialize_state(ctx)
            t = 0.0
            for _ in range(3):
                dt = api.compute_euler_dt(ctx, t)
                api.euler_fv_one_step(ctx, dt, t)
                t += dt
            ms = []
            for k in range(steps):
                dt = api.compute_euler_dt(ctx, t)
                with torch.cuda.stream(stream):
                    flush.fill_(float(k))
                    sink.copy_(flush.sum())
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                _lib.check(lib.ecg_euler_fv_one_step(ctx.handle, dt, t, None), "euler_fv_one_step")
                b.record(stream)
                b.synchronize()
                ms.append(a.elapsed_time(b))
                t += dt
            d = api.compute_diagnostics(ctx)
        us = 1e3 * sum(ms) / len(ms)
        gbs = BYTES_PER_CELL * cells / (us * 1e-6) / 1e9
        res.append({"workload": name, "cells": cells, "us_per_step": us, "value": cells / (us * 1e-6), "unit": UNIT,
                    "achieved_gbs": gbs, "hbm_frac": gbs / peak,
                    "state_ok": bool(d.nonfinite_count == 0 and d.rho_min > 0 and d.pressure_min > 0)})
    return {"steps_timed": steps, "cases": res}


def batch_leg(dev, stream, steps=200):
    """64 independent explicit O2 HLLC Riemann solves on the seeded grid ladder
    {64x64, 128x32, 256x256, 512x128, 1024x256}, one persistent launch per
    step for the whole batch, CUDA graphs; cell-updates/s over `steps` steps,
    timed with CUDA events on the batch's stream."""
    import torch

    from amrex_euler_allmach_explicit_imex_b200 import api, workloads

    cfgs, states = workloads.riemann_batch(64, seed=0)
    cells = sum(c.cfg.n_cell[0] * c.cfg.n_cell[1] for c in cfgs)
    with api.Batch(cfgs, device=dev.index or 0, stream=stream.cuda_stream) as b:
        for k, u in enumerate(states):
            b.upload(k, u)
        b.run(24)  # autotune and graph capture
        for k, u in enumerate(states):
            b.upload(k, u)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = b.run(steps)
        e1.record(stream)
        e1.synchronize()
        el = e0.elapsed_time(e1) * 1e-3
    ok = all(r.steps == steps and r.failed == 0 for r in res)
    peak, _ = peaks()
    return {"workload": "64 Riemann solves, grids drawn (seed 0) from 64x64..1024x256, O2 HLLC FP64, CFL 0.5",
            "cells": cells, "steps": steps, "seconds": el, "value": cells * steps / el, "unit": UNIT,
            "hbm_frac": BYTES_PER_CELL * cells * steps / el / 1e9 / peak, "all_solves_completed": ok}


def run_slab(args):
    """--slab: ONE grid (--slab-grid, default 10240x2560 of the bubble
    problem) split over the N ranks as x-slabs (slab.SlabSolver): every step
    packs the edge columns, swaps them with the neighbours over NCCL, steps
    each slab and takes the global dt as the minimum over ranks.  Strong
    scaling: value = the whole grid's cell-updates / (max over ranks of the
    event-timed region), which includes the halo exchange and the dt
    all-reduce."""
    import torch

    from amrex_euler_allmach_explicit_imex_b200 import slab
    from amrex_euler_allmach_explicit_imex_b200.config import read_config

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = init_dist(world, "nccl")
    dev = torch.device("cuda", local)
    nx, ny = (int(v) for v in args.slab_grid.lower().split("x"))
    kv = dict(WORKLOAD_KV, **{"amr.n_cell": f"{nx} {ny}"})
    cfg = read_config(kv).cfg
    solver = slab.SlabSolver(cfg, device=local, arith="fast")
    solver.initialize_state()
    t = 0.0
    for _ in range(args.warmup):
        dt = solver.compute_euler_dt(t)
        solver.euler_fv_one_step(dt, t)
        t += dt
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    stream = solver.stream
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        dt = solver.compute_euler_dt(t)
        solver.euler_fv_one_step(dt, t)
        t += dt
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = max_over_ranks(dist, e0.elapsed_time(e1), dev)
    cells = nx * ny
    value = cells * args.steps / (ms * 1e-3)
    d = solver.ctx.download()
    ok = bool(np.isfinite(d).all())
    solver.close()
    if rank == 0:
        peak, _ = peaks()
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (the shock-density bubble's initializer)",
                "config": {"workload": f"shock_density_bubble_2d {nx}x{ny}, explicit O2 HLLC, FP64, one grid in "
                                       f"{world} x-slabs with a 2-column NCCL halo exchange per step",
                           "grid": [nx, ny], "parallelism": f"slabs{world}"},
                "hbm_frac_per_gpu": BYTES_PER_CELL * cells / world / (ms / args.steps * 1e-3) / 1e9 / peak,
                "state_ok": ok}
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_ours(args):
    import torch

    from amrex_euler_allmach_explicit_imex_b200 import _lib, api
    from amrex_euler_allmach_explicit_imex_b200.config import read_config

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = init_dist(world, "nccl")
    dev = torch.device("cuda", local)
    lib = _lib.load()

    cfg = read_config(WORKLOAD_KV).cfg
    stream = torch.cuda.Stream(device=dev)
    ctx = api.Context(cfg, arith="fast", device=local, stream=stream.cuda_stream)
    # the problem's initial condition, written on the device (initialize_state)
    api.initialize_state(ctx)
    u0 = ctx.download()  # host copy for the end-to-end leg
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    flush_sink = torch.empty((), dtype=torch.float32, device=dev)
    cells = NX * NY
    fp64_peak = api.measure_fp64_peak(local)  # TFLOP/s on this GPU, before the timed region

    def one_step(t):
        dt = api.compute_euler_dt(ctx, t)
        api.euler_fv_one_step(ctx, dt, t)
        return t + dt

    # ---- device-resident throughput -----------------------------------------------------
    t = 0.0
    for _ in range(args.warmup):
        t = one_step(t)
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    dts = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize(dev)
        for k in range(args.steps):
            dt = api.compute_euler_dt(ctx, t)  # host read of the previous step's fused CFL reduction
            with torch.cuda.stream(stream):
                # write then read 256 MiB: no line of the state stays in L2,
                # and no dirty line is left for the step to write back; the
                # step is queued behind the flush, so the events time the
                # kernel, not the host's launch of it
                flush.fill_(float(k))
                flush_sink.copy_(flush.sum())
            ev[k][0].record(stream)
            # the C entry point without the degenerate-count read-back: the
            # events bracket the step's launch alone, not a host round trip
            _lib.check(lib.ecg_euler_fv_one_step(ctx.handle, dt, t, None), "euler_fv_one_step")
            ev[k][1].record(stream)
            dts.append(dt)
            t += dt
        torch.cuda.synchronize(dev)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    if dist is not None:
        dist.barrier()
    total_ms = max_over_ranks(dist, total_ms, dev)
    value = sum_over_ranks(dist, cells * args.steps, dev) / (total_ms * 1e-3)
    kern_s = (total_ms / args.steps) * 1e-3
    achieved = BYTES_PER_CELL * cells / kern_s / 1e9
    peak, peak_kind = peaks()
    d = api.compute_diagnostics(ctx)
    ok = d.nonfinite_count == 0 and d.rho_min > 0 and d.pressure_min > 0

    # ---- end to end through the C ABI with host buffers ----------------------------------
    # The driver's host-MultiFab sequence, one call per step
    # (ecg_euler_fv_one_step_host): this step's input crosses to the device and
    # its result comes back inside the timed region, pipelined over row bands;
    # dt is compute_euler_dt of the input (the fused reduction of the previous
    # step, whose result is that input).
    host_a = torch.from_numpy(u0).pin_memory()
    host_b = torch.empty_like(host_a).pin_memory()
    e2e_k = max(3, min(args.steps, 10))
    _lib.check(lib.ecg_upload_state(ctx.handle, host_a.data_ptr(), 0, 0, NX, NX * NY), "upload")
    te = 0.0
    deg = C.c_int32()
    # untimed warm-up calls: the first one creates the copy streams and events
    for _ in range(3):
        dt = api.compute_euler_dt(ctx, te)
        _lib.check(lib.ecg_euler_fv_one_step_host(ctx.handle, host_a.data_ptr(), host_b.data_ptr(), 0, 0, NX, NX * NY,
                                                  dt, te, C.byref(deg)), "euler_fv_one_step_host")
        host_a, host_b = host_b, host_a
        te += dt
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(e2e_k):
        dt = api.compute_euler_dt(ctx, te)
        _lib.check(lib.ecg_euler_fv_one_step_host(ctx.handle, host_a.data_ptr(), host_b.data_ptr(), 0, 0, NX, NX * NY,
                                                  dt, te, C.byref(deg)), "euler_fv_one_step_host")
        host_a, host_b = host_b, host_a
        te += dt
    e_end.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = max_over_ranks(dist, e_start.elapsed_time(e_end), dev)
    e2e_value = sum_over_ranks(dist, cells * e2e_k, dev) / (e2e_ms * 1e-3)

    # The same calls on pageable host memory (an FArrayBox as AMReX allocates
    # it, never registered with CUDA): the library copies each band through
    # its own pinned stage on host threads while the previous band crosses
    # (the first call allocates the stage; the warm-up calls cover it).
    page_a = np.ascontiguousarray(host_a.numpy()).copy()
    page_b = np.empty_like(page_a)
    for _ in range(2):
        dt = api.compute_euler_dt(ctx, te)
        _lib.check(lib.ecg_euler_fv_one_step_host(ctx.handle, page_a.ctypes.data, page_b.ctypes.data, 0, 0, NX,
                                                  NX * NY, dt, te, C.byref(deg)), "euler_fv_one_step_host")
        page_a, page_b = page_b, page_a
        te += dt
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    e_start.record(stream)
    for _ in range(e2e_k):
        dt = api.compute_euler_dt(ctx, te)
        _lib.check(lib.ecg_euler_fv_one_step_host(ctx.handle, page_a.ctypes.data, page_b.ctypes.data, 0, 0, NX,
                                                  NX * NY, dt, te, C.byref(deg)), "euler_fv_one_step_host")
        page_a, page_b = page_b, page_a
        te += dt
    e_end.record(stream)
    torch.cuda.synchronize(dev)
    pg_ms = max_over_ranks(dist, e_start.elapsed_time(e_end), dev)
    pg_value = sum_over_ranks(dist, cells * e2e_k, dev) / (pg_ms * 1e-3)

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            v, kind, cores, sample = cpu_reference_step_rate(args.cpu_steps, os.cpu_count())
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
        prof = step_profile()
        traffic = prof.get("dram_bytes_per_launch")
        fpc = prof.get("fp64_flop_per_cell")
        fp64 = None
        if fpc:
            got = fpc * cells / kern_s / 1e12
            fp64 = {"achieved": got, "peak": fp64_peak, "unit": "TFLOP/s", "frac": got / fp64_peak if fp64_peak else None,
                    "flop_per_cell": fpc, "peak_source": "ecg_measure_fp64_peak on this GPU (independent FMA chains)",
                    "note": "FP64 flops per cell from the ncu opcode counts of the step kernel (2 DFMA + DMUL + DADD)"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the shock-density-bubble initial condition of the reference's initialize_state, written on the device)", "config": CONFIG,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_source": peak_kind, "fp64": fp64,
                         "note": "algorithmic bytes = 64 B x 1,638,400 cells per launch; event time of the fused step kernel"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 32 * cells,
                    "d2h_bytes_per_step": 32 * cells, "host_memory": "pinned"},
            "e2e_pageable": {"value": pg_value, "unit": UNIT, "h2d_bytes_per_step": 32 * cells,
                             "d2h_bytes_per_step": 32 * cells, "host_memory": "pageable (numpy)"},
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "state_ok": bool(ok),
        }
        if world == 1 and not args.no_extra_legs:
            line["imex"] = imex_leg(dev, stream)
            line["hllcp"] = hllcp_leg(dev, stream)
            line["batched"] = batch_leg(dev, stream)
        print(json.dumps(line))
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=12)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra-legs", action="store_true", help="skip the IMEX and batched measurements")
    ap.add_argument("--slab", action="store_true",
                    help="strong scaling: one grid split over the ranks as x-slabs with an NCCL halo exchange")
    ap.add_argument("--slab-grid", default="10240x2560")
    ap.add_argument("--imex-case", type=int, default=None,
                    help="with --only imex: run the IMEX_CASES entry of this index alone")
    ap.add_argument("--only", choices=["imex", "batched", "hllcp"], default=None,
                    help="run one of the extra legs alone (profiling) and print its JSON")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.slab:
        return run_slab(args)
    if args.only:
        import torch

        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        stream = torch.cuda.Stream(device=dev)
        legs = {"imex": lambda: imex_leg(dev, stream, steps=2, only_case=args.imex_case),
                "batched": lambda: batch_leg(dev, stream),
                "hllcp": lambda: hllcp_leg(dev, stream)}
        leg = legs[args.only]()
        print(json.dumps({"leg": args.only, **leg}))
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
