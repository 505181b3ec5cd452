"""Python mirror of the reference's hot-path interface, on the CUDA library.

The reference's calls (amrex/apps/euler_compare/src/euler_compare/, all
inside one translation unit) and their counterparts here:

    euler_fv_one_step(state, geom, cfg, dt, time)         -> euler_fv_one_step(ctx, dt, time)
        numerics/explicit_update.hpp:58-102
    compute_euler_dt(state, geom, cfg, time)               -> compute_euler_dt(ctx, time)
        numerics/diagnostic_metrics_timestep.hpp:227-260
    compute_imex_dt(state, geom, cfg, time, diag)          -> compute_imex_dt(ctx, time)
        numerics/diagnostic_metrics_timestep.hpp:272-326
    compute_diagnostics(state, cfg)                        -> compute_diagnostics(ctx)
        numerics/diagnostic_metrics_timestep.hpp:18-47
    compute_admissibility_diagnostics(state, cfg)          -> compute_admissibility_diagnostics(ctx)
        numerics/diagnostic_metrics_timestep.hpp:49-111
    fill_problem_ghosts(state, geom, cfg, time)            -> fill_problem_ghosts(ctx, time)
        problems/boundary_conditions.hpp:202-219
    euler_imex_bdltv20_o1_source_map_picard_one_step(...)  -> euler_imex_bdltv20_o1_source_map_picard_one_step(ctx, dt)
        imex/imex_source_map_step.hpp:300-616

The MultiFab becomes a Context holding the device state; numpy arrays of
shape (4, ny, nx) (components rho, mx, my, E) move it in and out.
"""
import ctypes as C
import os

import numpy as np

from . import abi
from ._lib import EcgError, check, load
from .config import RunSettings, read_config


# cudaStreamLegacy: the legacy default stream, which torch's default stream is
_LEGACY_STREAM = 1


def gpu_options(arith="fast", imex_precision="fp64", device=0, tile_y=0, stream=None, **kw):
    """ecg_gpu_options.  stream: None for a context-owned stream, or a
    cudaStream_t handle; 0 (torch's default stream) selects the legacy default
    stream, so the context's work is ordered with torch's default-stream work."""
    lib = load()
    o = abi.GpuOptions()
    lib.ecg_default_gpu_options(C.byref(o))
    o.device = device
    o.arith = abi.ARITH_EXACT if arith == "exact" else abi.ARITH_FAST
    o.imex_precision = abi.IMEX_MIXED if imex_precision == "mixed" else abi.IMEX_FP64
    o.tile_y = tile_y
    o.stream = _LEGACY_STREAM if stream == 0 else stream
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Context:
    """One device-resident state (the MultiFab of the reference) and its
    configuration; owns all device buffers."""

    def __init__(self, cfg, slab=None, **gpu):
        """slab=(x0, x1, halo_lo, halo_hi): columns [x0, x1) of the grid, with
        ghost columns from neighbour slabs on the halo sides (ecg_create_slab)."""
        lib = load()
        if isinstance(cfg, RunSettings):
            cfg = cfg.cfg
        elif not isinstance(cfg, abi.RunConfig):
            cfg = read_config(cfg).cfg
        self.cfg = cfg.copy()
        self.opt = gpu_options(**gpu)
        h = C.c_void_p()
        if slab is None:
            check(lib.ecg_create(C.byref(h), C.byref(self.cfg), C.byref(self.opt)), "ecg_create")
            self.nx = self.cfg.n_cell[0]
        else:
            x0, x1, hlo, hhi = slab
            check(lib.ecg_create_slab(C.byref(h), C.byref(self.cfg), C.byref(self.opt), int(x0), int(x1), int(bool(hlo)),
                                      int(bool(hhi))), "ecg_create_slab")
            self.nx = int(x1) - int(x0)
        self._h = h
        self.ny = self.cfg.n_cell[1]

    def bind_halo(self, lo, hi):
        """Device halo blocks (torch tensors of 8 ny float64, or None) the
        steps of a slab read (ecg_slab_bind_halo)."""
        check(load().ecg_slab_bind_halo(self._h, None if lo is None else lo.data_ptr(),
                                        None if hi is None else hi.data_ptr()), "ecg_slab_bind_halo", self._h)

    def pack(self, lo, hi):
        """The slab's edge columns into device blocks (ecg_slab_pack)."""
        check(load().ecg_slab_pack(self._h, None if lo is None else lo.data_ptr(), None if hi is None else hi.data_ptr()),
              "ecg_slab_pack", self._h)

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            load().ecg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- state exchange (Array4 description of a numpy array) ----
    def upload(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.shape != (4, self.ny, self.nx):
            raise ValueError(f"state shape {u.shape} != (4, {self.ny}, {self.nx})")
        check(load().ecg_upload_state(self._h, u.ctypes.data, 0, 0, self.nx, self.nx * self.ny), "upload", self._h)

    def download(self, out=None):
        if out is None:
            out = np.empty((4, self.ny, self.nx), dtype=np.float64)
        check(load().ecg_download_state(self._h, out.ctypes.data, 0, 0, self.nx, self.nx * self.ny), "download",
              self._h)
        return out

    def upload_device(self, ptr, lo=(0, 0), jstride=None, nstride=None):
        jstride = self.nx if jstride is None else jstride
        nstride = jstride * self.ny if nstride is None else nstride
        check(load().ecg_upload_state_device(self._h, ptr, lo[0], lo[1], jstride, nstride), "upload_device", self._h)

    def download_device(self, ptr, lo=(0, 0), jstride=None, nstride=None):
        jstride = self.nx if jstride is None else jstride
        nstride = jstride * self.ny if nstride is None else nstride
        check(load().ecg_download_state_device(self._h, ptr, lo[0], lo[1], jstride, nstride), "download_device",
              self._h)

    def synchronize(self):
        check(load().ecg_synchronize(self._h), "synchronize", self._h)


def initialize_state(ctx):
    """initialize_state (problems/problem_initialization.hpp:420-435) on the device."""
    check(load().ecg_initialize_state(ctx.handle), "initialize_state", ctx.handle)


def euler_fv_one_step(ctx, dt, time=0.0):
    """One explicit step; returns the HLLC degenerate-star count."""
    n = C.c_int32()
    check(load().ecg_euler_fv_one_step(ctx.handle, dt, time, C.byref(n)), "euler_fv_one_step", ctx.handle)
    return n.value


def euler_fv_one_step_host(ctx, u_in, u_out, dt, time=0.0):
    """One explicit step of a host state (numpy (4, ny, nx) float64 arrays,
    preferably in pinned memory): upload, step and download pipelined over
    row bands (ecg_euler_fv_one_step_host).  Returns the degenerate count."""
    ny, nx = ctx.ny, ctx.nx
    for a in (u_in, u_out):
        if a.shape != (4, ny, nx) or a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError("host states must be C-contiguous float64 arrays of shape (4, ny, nx)")
    n = C.c_int32()
    check(load().ecg_euler_fv_one_step_host(ctx.handle, u_in.ctypes.data, u_out.ctypes.data, 0, 0, nx, nx * ny, dt,
                                            time, C.byref(n)), "euler_fv_one_step_host", ctx.handle)
    return n.value


def compute_euler_dt(ctx, time=0.0):
    dt = C.c_double()
    check(load().ecg_compute_euler_dt(ctx.handle, time, C.byref(dt)), "compute_euler_dt", ctx.handle)
    return dt.value


def compute_imex_dt(ctx, time=0.0):
    dt = C.c_double()
    d = abi.ImexTimestepDiag()
    check(load().ecg_compute_imex_dt(ctx.handle, time, C.byref(dt), C.byref(d)), "compute_imex_dt", ctx.handle)
    return dt.value, d


def compute_diagnostics(ctx):
    d = abi.Diagnostics()
    check(load().ecg_compute_diagnostics(ctx.handle, C.byref(d)), "compute_diagnostics", ctx.handle)
    return d


def compute_admissibility_diagnostics(ctx):
    d = abi.Admissibility()
    check(load().ecg_compute_admissibility_diagnostics(ctx.handle, C.byref(d)), "compute_admissibility_diagnostics",
          ctx.handle)
    return d


def fill_problem_ghosts(ctx, time=0.0):
    """The ghosted box (4, ny+4, nx+4) as fill_problem_ghosts leaves it."""
    g = np.empty((4, ctx.ny + 4, ctx.nx + 4), dtype=np.float64)
    check(load().ecg_fill_problem_ghosts(ctx.handle, time, g.ctypes.data), "fill_problem_ghosts", ctx.handle)
    return g


def euler_imex_bdltv20_o1_source_map_picard_one_step(ctx, dt):
    """The IMEX T1/S2 step; returns the diagnostics record.  The state is
    updated only when the solve converged (as in the reference)."""
    d = abi.ImexDiag()
    check(load().ecg_imex_step(ctx.handle, dt, C.byref(d)), "imex step", ctx.handle)
    return d


def solver_status_str(code):
    return load().ecg_solver_status_str(code).decode()


def run(ctx, max_step, stop_time):
    """The driver's time loop on the device; returns a RunResult."""
    r = abi.RunResult()
    check(load().ecg_run(ctx.handle, max_step, stop_time, C.byref(r)), "run", ctx.handle)
    return r


def paper_options(settings):
    """ecg_paper_options from the euler.bdltv20_paper_* settings of a run
    (core/run_config.hpp:33-52: dt -1 = eq79 CFL mode, epsilon 1, 4096 steps)."""
    mode = settings.bdltv20_paper_t1_s2
    if mode not in abi.PAPER_MODE:
        raise ValueError("Unsupported euler.bdltv20_paper_t1_s2 setting.")
    o = abi.PaperOptions()
    o.mode = abi.PAPER_MODE[mode]
    o.fixed_dt = float(settings.extra.get("bdltv20_paper_t1_s2_dt", -1.0))
    o.epsilon = float(settings.extra.get("bdltv20_paper_epsilon", 1.0))
    o.max_steps = int(settings.extra.get("bdltv20_paper_t1_s2_max_steps", 4096))
    return o


def run_bdltv20_paper_t1_s2(ctx, settings):
    """run_bdltv20_paper_t1_s2 (imex/imex_bdltv20_direct_driver.hpp:44-779) on the
    device: initialises the context from its problem, runs the direct T1/S2
    driver, and returns its report (abi.PaperResult)."""
    o = paper_options(settings)
    r = abi.PaperResult()
    check(load().ecg_paper_t1s2_run(ctx.handle, C.byref(o), C.byref(r)), "run_bdltv20_paper_t1_s2", ctx.handle)
    return r


def write_final_csv(ctx, path, step, time, trial_minima=(float("nan"),) * 3):
    """The problem's final CSV (write_gresho_final_csv, write_toro_final_csv,
    write_riemann_quadrant_final_csv or write_advection_blob_final_csv,
    io/output_cases.hpp:16-216) of the context's state."""
    info = abi.OutputInfo()
    info.step, info.time = int(step), float(time)
    info.trial_density_min, info.trial_pressure_min, info.trial_internal_energy_min = map(float, trial_minima)
    check(load().ecg_write_final_csv(ctx.handle, os.fsencode(path), C.byref(info)), "write_final_csv", ctx.handle)


def shock_bubble_metrics(ctx, time=0.0):
    """compute_shock_density_bubble_metrics (io/output_cases.hpp:329-403)."""
    m = abi.BubbleMetrics()
    check(load().ecg_shock_bubble_metrics(ctx.handle, float(time), C.byref(m)), "shock_bubble_metrics", ctx.handle)
    return m


def write_bubble_snapshot(ctx, directory, index, step, time, asynchronous=False):
    """write_shock_density_bubble_snapshot (io/output_cases.hpp:405-487); with
    asynchronous=True the file is written by a host thread while stepping
    goes on (output_wait joins)."""
    check(load().ecg_write_bubble_snapshot(ctx.handle, os.fsencode(directory), int(index), int(step), float(time),
                                           1 if asynchronous else 0), "write_bubble_snapshot", ctx.handle)


def output_wait(ctx):
    """Joins the asynchronous snapshot writers."""
    failed = C.c_int32()
    check(load().ecg_output_wait(ctx.handle, C.byref(failed)), "output_wait", ctx.handle)


def write_bubble_summary_csv(ctx, path, steps_accepted, time, status="ok", failure_category="ok", steps_rejected=0,
                             wall_time_sec=0.0, dt_min=float("nan"), dt_max=float("nan"), dt_mean=float("nan"),
                             snapshot_status="not_requested", snapshot_dir="",
                             snapshot_times="0,0.06,0.12,0.18,0.24,0.30"):
    """write_shock_density_bubble_summary_csv (io/output_cases.hpp:489-588)."""
    r = abi.BubbleRun()
    r.steps_accepted, r.steps_rejected, r.time = int(steps_accepted), int(steps_rejected), float(time)
    r.wall_time_sec, r.dt_min, r.dt_max, r.dt_mean = map(float, (wall_time_sec, dt_min, dt_max, dt_mean))
    r.status, r.failure_category, r.snapshot_status = status.encode(), failure_category.encode(), snapshot_status.encode()
    r.snapshot_dir, r.snapshot_times = snapshot_dir.encode(), snapshot_times.encode()
    check(load().ecg_write_bubble_summary_csv(ctx.handle, os.fsencode(path), C.byref(r)), "write_bubble_summary_csv",
          ctx.handle)


def measure_fp64_peak(device=0):
    """FP64 FMA throughput of `device` in TFLOP/s (ecg_measure_fp64_peak): the
    denominator of the explicit step's FP64 roofline."""
    v = C.c_double()
    check(load().ecg_measure_fp64_peak(device, C.byref(v)), "measure_fp64_peak")
    return v.value


def check_grid_barrier_timeout(spin_limit=4096, device=0):
    """The GMRES grid barrier's bounded wait (ecg_check_grid_barrier_timeout):
    returns (blocks that passed the first barrier, blocks whose wait at the
    second ran out); (4, 3) when the bound works."""
    first, out = C.c_int32(), C.c_int32()
    check(load().ecg_check_grid_barrier_timeout(device, spin_limit, C.byref(first), C.byref(out)),
          "check_grid_barrier_timeout")
    return first.value, out.value


class Batch:
    """Many independent explicit solves of uneven grid sizes advanced together
    (ecg_batch_*): one persistent launch per step for the whole batch, CUDA
    graphs of 24 steps, dt per solve on the device."""

    def __init__(self, cfgs, **gpu):
        lib = load()
        cfgs = [c.cfg if isinstance(c, RunSettings) else (c if isinstance(c, abi.RunConfig) else read_config(c).cfg)
                for c in cfgs]
        self.n = len(cfgs)
        self.cfgs = (abi.RunConfig * self.n)(*[c.copy() for c in cfgs])
        self.opt = gpu_options(**gpu)
        h = C.c_void_p()
        code = lib.ecg_batch_create(C.byref(h), self.n, self.cfgs, C.byref(self.opt))
        if code != 0:
            raise EcgError(code, "ecg_batch_create: " + lib.ecg_status_str(code).decode())
        self._h = h
        self.shapes = [(c.n_cell[1], c.n_cell[0]) for c in cfgs]

    def _check(self, code, what):
        if code != 0:
            lib = load()
            raise EcgError(code, f"{what}: {lib.ecg_status_str(code).decode()}: {lib.ecg_batch_last_error(self._h).decode()}")

    def upload(self, k, u):
        ny, nx = self.shapes[k]
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.shape != (4, ny, nx):
            raise ValueError(f"state shape {u.shape} != (4, {ny}, {nx})")
        self._check(load().ecg_batch_upload(self._h, k, u.ctypes.data, 0, 0, nx, nx * ny), "batch upload")

    def download(self, k):
        ny, nx = self.shapes[k]
        out = np.empty((4, ny, nx), dtype=np.float64)
        self._check(load().ecg_batch_download(self._h, k, out.ctypes.data, 0, 0, nx, nx * ny), "batch download")
        return out

    def run(self, steps):
        """Advances every solve by up to `steps` steps; returns one BatchResult per solve."""
        res = (abi.BatchResult * self.n)()
        self._check(load().ecg_batch_run(self._h, steps, res), "batch run")
        return list(res)

    def close(self):
        if getattr(self, "_h", None):
            load().ecg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


__all__ = [
    "Batch",
    "Context",
    "EcgError",
    "check_grid_barrier_timeout",
    "compute_admissibility_diagnostics",
    "compute_diagnostics",
    "compute_euler_dt",
    "compute_imex_dt",
    "euler_fv_one_step",
    "euler_fv_one_step_host",
    "euler_imex_bdltv20_o1_source_map_picard_one_step",
    "fill_problem_ghosts",
    "gpu_options",
    "initialize_state",
    "measure_fp64_peak",
    "read_config",
    "run",
    "run_bdltv20_paper_t1_s2",
    "solver_status_str",
]
