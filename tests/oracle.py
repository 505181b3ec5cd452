"""Loaders for the CPU checkers under oracle/ (test infrastructure only).

Oracle      -- oracle/libecg_oracle.so, the C++ restatement of the reference
               algorithm (always built from this repository).
RefOracle   -- oracle/_ref/libecg_ref.so, the reference's own headers compiled
               against a single-box AMReX shim; present only where it was built
               (it needs the reference sources at build time).

Arrays are numpy float64 of shape (4, ny, nx): component planes rho, mx, my, E.
"""
import ctypes as C
import os

import numpy as np

from amrex_euler_allmach_explicit_imex_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "libecg_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libecg_ref.so")

_D = C.c_double
_P = C.c_void_p
_I = C.c_int
_CFG = C.POINTER(abi.RunConfig)


def _ptr(a):
    return a.ctypes.data_as(_P)


def _state(cfg):
    return np.zeros((4, cfg.n_cell[1], cfg.n_cell[0]), dtype=np.float64)


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        lib = C.CDLL(path)
        lib.ecgo_default_run_config.argtypes = [_CFG]
        lib.ecgo_initialize_state.argtypes = [_CFG, _P]
        lib.ecgo_fill_problem_ghosts.argtypes = [_CFG, _P, _D, _P]
        lib.ecgo_euler_fv_one_step.argtypes = [_CFG, _P, _D, _D]
        lib.ecgo_compute_euler_dt.argtypes = [_CFG, _P, _D]
        lib.ecgo_compute_euler_dt.restype = _D
        lib.ecgo_compute_imex_dt.argtypes = [_CFG, _P, _D, C.POINTER(abi.ImexTimestepDiag)]
        lib.ecgo_compute_imex_dt.restype = _D
        lib.ecgo_compute_diagnostics.argtypes = [_CFG, _P, C.POINTER(abi.Diagnostics)]
        lib.ecgo_compute_admissibility.argtypes = [_CFG, _P, C.POINTER(abi.Admissibility)]
        lib.ecgo_imex_step.argtypes = [_CFG, _P, _D, C.POINTER(abi.ImexDiag)]
        lib.ecgo_gmres_csr.argtypes = [_I, _P, _P, _P, _P, _P, _I, _D, _P] + [C.POINTER(_I)] * 4 + [C.POINTER(_D)] * 2
        lib.ecgo_run_explicit.argtypes = [_CFG, _P, _I, _D, C.POINTER(abi.RunResult)]
        lib.ecgo_exact_riemann_sample.argtypes = [_D, _D, _P, _P, _D, _D, _P]
        lib.ecgo_imex_build_system.argtypes = [_CFG, _P, _P, _P, _D, _P, _P, _P, _P, _I, C.POINTER(_I)]
        lib.ecgo_imex_star.argtypes = [_CFG, _P, _D, _P]
        lib.ecgo_corrected_momentum.argtypes = [_CFG, _P, _P, _D, _P]
        lib.ecgo_gresho_state.argtypes = [_CFG, _D, _D, _P]
        lib.ecgo_gresho_density_l1.argtypes = [_CFG, _P]
        lib.ecgo_gresho_density_l1.restype = _D
        self.lib = lib

    def default_config(self):
        c = abi.RunConfig()
        self.lib.ecgo_default_run_config(C.byref(c))
        return c

    def initialize(self, cfg):
        u = _state(cfg)
        self.lib.ecgo_initialize_state(C.byref(cfg), _ptr(u))
        return u

    def fill_ghosts(self, cfg, u, time=0.0):
        u = np.ascontiguousarray(u, dtype=np.float64)
        g = np.zeros((4, cfg.n_cell[1] + 4, cfg.n_cell[0] + 4))
        self.lib.ecgo_fill_problem_ghosts(C.byref(cfg), _ptr(u), time, _ptr(g))
        return g

    def step(self, cfg, u, dt, time=0.0):
        u = np.array(u, dtype=np.float64, order="C", copy=True)
        n = self.lib.ecgo_euler_fv_one_step(C.byref(cfg), _ptr(u), dt, time)
        return u, n

    def euler_dt(self, cfg, u, time=0.0):
        u = np.ascontiguousarray(u, dtype=np.float64)
        return self.lib.ecgo_compute_euler_dt(C.byref(cfg), _ptr(u), time)

    def imex_dt(self, cfg, u, time=0.0):
        u = np.ascontiguousarray(u, dtype=np.float64)
        d = abi.ImexTimestepDiag()
        dt = self.lib.ecgo_compute_imex_dt(C.byref(cfg), _ptr(u), time, C.byref(d))
        return dt, d

    def diagnostics(self, cfg, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        d = abi.Diagnostics()
        self.lib.ecgo_compute_diagnostics(C.byref(cfg), _ptr(u), C.byref(d))
        return d

    def admissibility(self, cfg, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        d = abi.Admissibility()
        self.lib.ecgo_compute_admissibility(C.byref(cfg), _ptr(u), C.byref(d))
        return d

    def imex_step(self, cfg, u, dt):
        u = np.array(u, dtype=np.float64, order="C", copy=True)
        d = abi.ImexDiag()
        self.lib.ecgo_imex_step(C.byref(cfg), _ptr(u), dt, C.byref(d))
        return u, d

    def gmres_csr(self, rp, col, val, b, x0, max_iter, tol):
        n = len(b)
        rp = np.ascontiguousarray(rp, dtype=np.int32)
        col = np.ascontiguousarray(col, dtype=np.int32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        x = np.zeros(n)
        it, cv, bd, nf = _I(), _I(), _I(), _I()
        rl, rr = _D(), _D()
        self.lib.ecgo_gmres_csr(n, _ptr(rp), _ptr(col), _ptr(val), _ptr(b), _ptr(x0), max_iter, tol, _ptr(x),
                                C.byref(it), C.byref(cv), C.byref(bd), C.byref(nf), C.byref(rl), C.byref(rr))
        return dict(x=x, iterations=it.value, converged=bool(cv.value), breakdown=bool(bd.value),
                    nonfinite=bool(nf.value), residual_linf=rl.value, relative_residual_linf=rr.value)

    def imex_star(self, cfg, u, dt):
        u = np.ascontiguousarray(u, dtype=np.float64)
        s = np.zeros_like(u)
        self.lib.ecgo_imex_star(C.byref(cfg), _ptr(u), dt, _ptr(s))
        return s

    def build_system(self, cfg, star, p, k, dt):
        n = star.shape[1] * star.shape[2]
        cap = 11 * n
        rp = np.zeros(n + 1, dtype=np.int32)
        col = np.zeros(cap, dtype=np.int32)
        val = np.zeros(cap)
        rhs = np.zeros(n)
        nf = _I()
        star = np.ascontiguousarray(star, dtype=np.float64)
        p = np.ascontiguousarray(p, dtype=np.float64)
        k = np.ascontiguousarray(k, dtype=np.float64)
        nnz = self.lib.ecgo_imex_build_system(C.byref(cfg), _ptr(star), _ptr(p), _ptr(k), dt, _ptr(rp), _ptr(col),
                                              _ptr(val), _ptr(rhs), cap, C.byref(nf))
        return rp, col[:nnz], val[:nnz], rhs, nf.value

    def corrected_momentum(self, cfg, star, p, dt):
        k = np.zeros((2, star.shape[1], star.shape[2]))
        self.lib.ecgo_corrected_momentum(C.byref(cfg), _ptr(np.ascontiguousarray(star)), _ptr(np.ascontiguousarray(p)),
                                         dt, _ptr(k))
        return k

    def run_explicit(self, cfg, u, max_step, stop_time):
        u = np.array(u, dtype=np.float64, order="C", copy=True)
        r = abi.RunResult()
        self.lib.ecgo_run_explicit(C.byref(cfg), _ptr(u), max_step, stop_time, C.byref(r))
        return u, r

    def exact_riemann(self, x, t, left, right, gamma, x0):
        l = np.asarray(left, dtype=np.float64)
        r = np.asarray(right, dtype=np.float64)
        out = np.zeros(4)
        self.lib.ecgo_exact_riemann_sample(x, t, _ptr(l), _ptr(r), gamma, x0, _ptr(out))
        return out

    def gresho_density_l1(self, cfg, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        return self.lib.ecgo_gresho_density_l1(C.byref(cfg), _ptr(u))


class RefOracle:
    """The reference's own code; configured from key=value text via its read_config()."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference is available")
        lib = C.CDLL(path)
        lib.ecref_paper_run.argtypes = [C.c_char_p, C.c_int]
        lib.ecref_write_final_csv.argtypes = [_P, C.c_int, _D, C.c_char_p, _D, _D, _D]
        lib.ecref_bubble_metrics.argtypes = [_P, _D, _P]
        lib.ecref_bubble_snapshot.argtypes = [_P, C.c_int, _D, C.c_int, C.c_char_p]
        lib.ecref_bubble_summary.argtypes = [_P, C.c_char_p, C.c_int, _D, C.c_char_p, C.c_char_p, C.c_int, _D, _D,
                                             _D, _D, C.c_char_p, C.c_char_p, C.c_char_p]
        lib.ecref_paper_run.restype = C.c_int
        lib.ecref_configure.argtypes = [C.c_char_p]
        lib.ecref_last_error.restype = C.c_char_p
        lib.ecref_get_config.argtypes = [_CFG]
        lib.ecref_initialize_state.argtypes = [_P]
        lib.ecref_euler_fv_one_step.argtypes = [_P, _D, _D]
        lib.ecref_compute_euler_dt.argtypes = [_P, _D]
        lib.ecref_compute_euler_dt.restype = _D
        lib.ecref_compute_imex_dt.argtypes = [_P, _D, C.POINTER(abi.ImexTimestepDiag)]
        lib.ecref_compute_imex_dt.restype = _D
        lib.ecref_compute_diagnostics.argtypes = [_P, C.POINTER(abi.Diagnostics)]
        lib.ecref_compute_admissibility.argtypes = [_P, C.POINTER(abi.Admissibility)]
        lib.ecref_fill_problem_ghosts.argtypes = [_P, _D, _P]
        lib.ecref_imex_step.argtypes = [_P, _D, C.POINTER(abi.ImexDiag)]
        lib.ecref_imex_star.argtypes = [_P, _D, _P]
        lib.ecref_imex_build_system.argtypes = [_P, _P, _P, _D, _P, _P, _P, _P, _I, C.POINTER(_I)]
        lib.ecref_gmres.argtypes = [_I, _P, _P, _P, _P, _P, _I, _D, _P] + [C.POINTER(_I)] * 4 + [C.POINTER(_D)] * 2
        lib.ecref_corrected_momentum.argtypes = [_P, _P, _D, _P]
        lib.ecref_exact_riemann_sample.argtypes = [_D, _D, _P, _P, _D, _D, _P]
        lib.ecref_gresho_density_l1.argtypes = [_P]
        lib.ecref_gresho_density_l1.restype = _D
        self.lib = lib
        self.cfg = None

    def configure(self, kv):
        text = kv if isinstance(kv, str) else "\n".join(f"{k}={v}" for k, v in kv.items())
        if self.lib.ecref_configure(text.encode()) != 0:
            raise ValueError(self.lib.ecref_last_error().decode())
        c = abi.RunConfig()
        self.lib.ecref_get_config(C.byref(c))
        self.cfg = c
        return c

    def paper_run(self):
        """The reference's direct T1/S2 driver on the configured run: (exit
        code, {key: value} of its report)."""
        buf = C.create_string_buffer(1 << 16)
        rc = self.lib.ecref_paper_run(buf, len(buf))
        rep = {}
        for line in buf.value.decode().splitlines():
            k, _, v = line.partition("=")
            rep[k.strip()] = v.strip()
        return rc, rep

    def write_final_csv(self, u, step, time, path, trial=(float("nan"),) * 3):
        """The reference's final CSV writer for the configured problem."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        rc = self.lib.ecref_write_final_csv(u.ctypes.data_as(_P), int(step), float(time), os.fsencode(path), *trial)
        if rc != 0:
            raise RuntimeError("ecref_write_final_csv failed")

    def bubble_metrics(self, u, time=0.0):
        """compute_shock_density_bubble_metrics: (nine values, nonfinite count)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.zeros(9)
        nf = self.lib.ecref_bubble_metrics(u.ctypes.data_as(_P), float(time), out.ctypes.data_as(_P))
        return out, nf

    def bubble_snapshot(self, u, step, time, index, directory):
        u = np.ascontiguousarray(u, dtype=np.float64)
        if self.lib.ecref_bubble_snapshot(u.ctypes.data_as(_P), int(step), float(time), int(index),
                                          os.fsencode(directory)) != 0:
            raise RuntimeError("ecref_bubble_snapshot failed")

    def bubble_summary(self, u, path, step, time, status, failure, rejected, wall, dt_min, dt_max, dt_mean,
                       snapshot_status, snapshot_dir, snapshot_times):
        u = np.ascontiguousarray(u, dtype=np.float64)
        self.lib.ecref_bubble_summary(u.ctypes.data_as(_P), os.fsencode(path), int(step), float(time), status.encode(),
                                      failure.encode(), int(rejected), float(wall), float(dt_min), float(dt_max),
                                      float(dt_mean), snapshot_status.encode(), snapshot_dir.encode(),
                                      snapshot_times.encode())

    def initialize(self):
        u = _state(self.cfg)
        if self.lib.ecref_initialize_state(_ptr(u)) != 0:
            raise ValueError(self.lib.ecref_last_error().decode())
        return u

    def step(self, u, dt, time=0.0):
        u = np.array(u, dtype=np.float64, order="C", copy=True)
        n = self.lib.ecref_euler_fv_one_step(_ptr(u), dt, time)
        return u, n

    def euler_dt(self, u, time=0.0):
        u = np.ascontiguousarray(u, dtype=np.float64)
        return self.lib.ecref_compute_euler_dt(_ptr(u), time)

    def imex_dt(self, u, time=0.0):
        u = np.ascontiguousarray(u, dtype=np.float64)
        d = abi.ImexTimestepDiag()
        dt = self.lib.ecref_compute_imex_dt(_ptr(u), time, C.byref(d))
        return dt, d

    def diagnostics(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        d = abi.Diagnostics()
        self.lib.ecref_compute_diagnostics(_ptr(u), C.byref(d))
        return d

    def admissibility(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        d = abi.Admissibility()
        self.lib.ecref_compute_admissibility(_ptr(u), C.byref(d))
        return d

    def fill_ghosts(self, u, time=0.0):
        u = np.ascontiguousarray(u, dtype=np.float64)
        g = np.zeros((4, self.cfg.n_cell[1] + 4, self.cfg.n_cell[0] + 4))
        self.lib.ecref_fill_problem_ghosts(_ptr(u), time, _ptr(g))
        return g

    def imex_step(self, u, dt):
        u = np.array(u, dtype=np.float64, order="C", copy=True)
        d = abi.ImexDiag()
        self.lib.ecref_imex_step(_ptr(u), dt, C.byref(d))
        return u, d

    def imex_star(self, u, dt):
        u = np.ascontiguousarray(u, dtype=np.float64)
        s = np.zeros_like(u)
        self.lib.ecref_imex_star(_ptr(u), dt, _ptr(s))
        return s

    def build_system(self, star, p, k, dt):
        n = star.shape[1] * star.shape[2]
        cap = 11 * n
        rp = np.zeros(n + 1, dtype=np.int32)
        col = np.zeros(cap, dtype=np.int32)
        val = np.zeros(cap)
        rhs = np.zeros(n)
        nf = _I()
        star = np.ascontiguousarray(star, dtype=np.float64)
        p = np.ascontiguousarray(p, dtype=np.float64)
        k = np.ascontiguousarray(k, dtype=np.float64)
        nnz = self.lib.ecref_imex_build_system(_ptr(star), _ptr(p), _ptr(k), dt, _ptr(rp), _ptr(col), _ptr(val),
                                               _ptr(rhs), cap, C.byref(nf))
        return rp, col[:nnz], val[:nnz], rhs, nf.value

    def gmres_csr(self, rp, col, val, b, x0, max_iter, tol):
        n = len(b)
        rp = np.ascontiguousarray(rp, dtype=np.int32)
        col = np.ascontiguousarray(col, dtype=np.int32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        x = np.zeros(n)
        it, cv, bd, nf = _I(), _I(), _I(), _I()
        rl, rr = _D(), _D()
        self.lib.ecref_gmres(n, _ptr(rp), _ptr(col), _ptr(val), _ptr(b), _ptr(x0), max_iter, tol, _ptr(x),
                             C.byref(it), C.byref(cv), C.byref(bd), C.byref(nf), C.byref(rl), C.byref(rr))
        return dict(x=x, iterations=it.value, converged=bool(cv.value), breakdown=bool(bd.value),
                    nonfinite=bool(nf.value), residual_linf=rl.value, relative_residual_linf=rr.value)

    def corrected_momentum(self, star, p, dt):
        k = np.zeros((2, star.shape[1], star.shape[2]))
        self.lib.ecref_corrected_momentum(_ptr(np.ascontiguousarray(star)), _ptr(np.ascontiguousarray(p)), dt, _ptr(k))
        return k

    def exact_riemann(self, x, t, left, right, gamma, x0):
        l = np.asarray(left, dtype=np.float64)
        r = np.asarray(right, dtype=np.float64)
        out = np.zeros(4)
        self.lib.ecref_exact_riemann_sample(x, t, _ptr(l), _ptr(r), gamma, x0, _ptr(out))
        return out

    def gresho_density_l1(self, u):
        return self.lib.ecref_gresho_density_l1(_ptr(np.ascontiguousarray(u, dtype=np.float64)))


def ref_available():
    return os.path.exists(REF_SO)
