"""The C-ABI library: loads without a GPU, exports every entry point that
include/ecg.h declares, and its structs match the ctypes mirror."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from amrex_euler_allmach_explicit_imex_b200 import _lib, abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ecg.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ecg_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_everything():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_host_only_entry_points():
    lib = _lib.load()
    assert lib.ecg_abi_version() == 1
    assert lib.ecg_status_str(0) == b"ok"
    assert [lib.ecg_solver_status_str(i).decode() for i in range(len(abi.SOLVER_STATUS))] == abi.SOLVER_STATUS
    c = abi.RunConfig()
    lib.ecg_default_run_config(C.byref(c))
    from amrex_euler_allmach_explicit_imex_b200.config import default_run_config

    assert c.as_dict() == default_run_config().as_dict()


def test_create_without_device_fails_cleanly():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    lib = _lib.load()
    cfg = abi.RunConfig()
    lib.ecg_default_run_config(C.byref(cfg))
    h = C.c_void_p()
    assert lib.ecg_create(C.byref(h), C.byref(cfg), None) == 4  # ECG_ERR_NO_DEVICE
    assert not h.value


STRUCTS = {
    "ecg_run_config": abi.RunConfig,
    "ecg_gpu_options": abi.GpuOptions,
    "ecg_diagnostics": abi.Diagnostics,
    "ecg_admissibility": abi.Admissibility,
    "ecg_imex_timestep_diag": abi.ImexTimestepDiag,
    "ecg_imex_diag": abi.ImexDiag,
    "ecg_run_result": abi.RunResult,
    "ecg_batch_result": abi.BatchResult,
}


def test_struct_layouts_match_header():
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"ecg.h\"\nint main(void){\n"
    for name, cls in STRUCTS.items():
        src += f'printf("{name} %zu\\n", sizeof({name}));\n'
        for field, _ in cls._fields_:
            src += f'printf("{name}.{field} %zu\\n", offsetof({name}, {field}));\n'
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        c_path = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c_path, "w").write(src)
        subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), c_path, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    got = dict(line.rsplit(" ", 1) for line in out.strip().splitlines())
    for name, cls in STRUCTS.items():
        assert int(got[name]) == C.sizeof(cls), name
        for field, _ in cls._fields_:
            assert int(got[f"{name}.{field}"]) == getattr(cls, field).offset, f"{name}.{field}"
