import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU and libecg.so")
    config.addinivalue_line("markers", "slow: longer CPU cases")


def _ensure_oracle():
    so = os.path.join(ROOT, "oracle", "libecg_oracle.so")
    src = os.path.join(ROOT, "oracle", "ecg_oracle.cpp")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


_ensure_oracle()


def gpu_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from tests.oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from tests.oracle import RefOracle, ref_available

    if not ref_available():
        pytest.skip("oracle/_ref not built here (needs the reference sources)")
    return RefOracle()


@pytest.fixture(scope="session")
def gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from amrex_euler_allmach_explicit_imex_b200 import _lib

    return _lib.load()
