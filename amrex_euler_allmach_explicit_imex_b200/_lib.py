"""Loads libecg.so (the CUDA hot path) through ctypes and declares its C ABI.

The library is built in-tree by build.py.  There is no CPU fallback: if the
library is missing or no sm_100 GPU is present, calls fail loudly.
"""
import ctypes as C
import os

from . import abi

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libecg.so")

_D = C.c_double
_P = C.c_void_p
_I32 = C.c_int32
_I64 = C.c_int64
_CTX = C.c_void_p

# every function include/ecg.h declares: name -> (restype, argtypes)
SIGNATURES = {
    "ecg_abi_version": (_I32, []),
    "ecg_status_str": (C.c_char_p, [C.c_int]),
    "ecg_solver_status_str": (C.c_char_p, [_I32]),
    "ecg_default_run_config": (None, [C.POINTER(abi.RunConfig)]),
    "ecg_default_gpu_options": (None, [C.POINTER(abi.GpuOptions)]),
    "ecg_create": (C.c_int, [C.POINTER(_CTX), C.POINTER(abi.RunConfig), C.POINTER(abi.GpuOptions)]),
    "ecg_destroy": (None, [_CTX]),
    "ecg_last_error": (C.c_char_p, [_CTX]),
    "ecg_upload_state": (C.c_int, [_CTX, _P, _I32, _I32, _I64, _I64]),
    "ecg_download_state": (C.c_int, [_CTX, _P, _I32, _I32, _I64, _I64]),
    "ecg_upload_state_device": (C.c_int, [_CTX, _P, _I32, _I32, _I64, _I64]),
    "ecg_download_state_device": (C.c_int, [_CTX, _P, _I32, _I32, _I64, _I64]),
    "ecg_fill_problem_ghosts": (C.c_int, [_CTX, _D, _P]),
    "ecg_synchronize": (C.c_int, [_CTX]),
    "ecg_initialize_state": (C.c_int, [_CTX]),
    "ecg_paper_t1s2_run": (C.c_int, [_CTX, C.POINTER(abi.PaperOptions), C.POINTER(abi.PaperResult)]),
    "ecg_measure_fp64_peak": (C.c_int, [C.c_int32, C.POINTER(C.c_double)]),
    "ecg_check_grid_barrier_timeout": (C.c_int, [C.c_int32, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "ecg_create_slab": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(abi.RunConfig), C.POINTER(abi.GpuOptions), C.c_int32,
                                  C.c_int32, C.c_int32, C.c_int32]),
    "ecg_slab_bind_halo": (C.c_int, [_CTX, C.c_void_p, C.c_void_p]),
    "ecg_slab_pack": (C.c_int, [_CTX, C.c_void_p, C.c_void_p]),
    "ecg_euler_fv_one_step_host": (C.c_int, [_CTX, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int64, C.c_int64,
                                             C.c_double, C.c_double, C.POINTER(C.c_int32)]),
    "ecg_write_final_csv": (C.c_int, [_CTX, C.c_char_p, C.POINTER(abi.OutputInfo)]),
    "ecg_shock_bubble_metrics": (C.c_int, [_CTX, C.c_double, C.POINTER(abi.BubbleMetrics)]),
    "ecg_write_bubble_snapshot": (C.c_int, [_CTX, C.c_char_p, C.c_int32, C.c_int32, C.c_double, C.c_int32]),
    "ecg_output_wait": (C.c_int, [_CTX, C.POINTER(C.c_int32)]),
    "ecg_write_bubble_summary_csv": (C.c_int, [_CTX, C.c_char_p, C.POINTER(abi.BubbleRun)]),
    "ecg_euler_fv_one_step": (C.c_int, [_CTX, _D, _D, C.POINTER(_I32)]),
    "ecg_compute_euler_dt": (C.c_int, [_CTX, _D, C.POINTER(_D)]),
    "ecg_compute_imex_dt": (C.c_int, [_CTX, _D, C.POINTER(_D), C.POINTER(abi.ImexTimestepDiag)]),
    "ecg_compute_diagnostics": (C.c_int, [_CTX, C.POINTER(abi.Diagnostics)]),
    "ecg_compute_admissibility_diagnostics": (C.c_int, [_CTX, C.POINTER(abi.Admissibility)]),
    "ecg_imex_step": (C.c_int, [_CTX, _D, C.POINTER(abi.ImexDiag)]),
    "ecg_run": (C.c_int, [_CTX, _I32, _D, C.POINTER(abi.RunResult)]),
    "ecg_explicit_step_vjp_device": (C.c_int, [_CTX, _P, _D, _P, _P]),
    "ecg_explicit_step_device": (C.c_int, [_CTX, _P, _D, _P]),
    "ecg_euler_fv_one_step_noalloc": (C.c_int, [C.POINTER(abi.RunConfig), C.POINTER(abi.GpuOptions), _P, _P, _I32,
                                                _I32, _I64, _I64, _D, _D, C.POINTER(_I32), C.c_char_p, _I32]),
    "ecg_batch_create": (C.c_int, [C.POINTER(_P), _I32, C.POINTER(abi.RunConfig), C.POINTER(abi.GpuOptions)]),
    "ecg_batch_destroy": (None, [_P]),
    "ecg_batch_upload": (C.c_int, [_P, _I32, _P, _I32, _I32, _I64, _I64]),
    "ecg_batch_download": (C.c_int, [_P, _I32, _P, _I32, _I32, _I64, _I64]),
    "ecg_batch_run": (C.c_int, [_P, _I32, C.POINTER(abi.BatchResult)]),
    "ecg_batch_last_error": (C.c_char_p, [_P]),
}

_lib = None


def load():
    """The loaded libecg.so; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m amrex_euler_allmach_explicit_imex_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class EcgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{msg} (status {code})")
        self.code = code


def check(code, what, ctx=None):
    if code != 0:
        lib = load()
        detail = lib.ecg_status_str(code).decode()
        if ctx:
            err = lib.ecg_last_error(ctx)
            if err:
                detail += ": " + err.decode()
        raise EcgError(code, f"{what}: {detail}")
