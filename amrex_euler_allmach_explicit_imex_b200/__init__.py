"""B200-native (sm_100a) euler_compare hot path.

The product is libecg.so (csrc/, built by build.py): hand-written FP64 CUDA
kernels behind the C ABI of include/ecg.h.  This package holds the ctypes
binding (_lib, abi), the reference-facing Python interface (api), the
ParmParse-style configuration reader (config), and the torch integration
(adjoint).
"""
from . import abi  # noqa: F401
from .config import ConfigError, RunSettings, read_config  # noqa: F401

__all__ = ["abi", "read_config", "RunSettings", "ConfigError"]
