"""Readers for the committed golden fixtures (generated by tests/golden/make_golden.py
from the reference's own code)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def kv_of(arr):
    return str(arr[()])


def explicit_cases():
    z = load("explicit_cases.npz")
    n = int(z["count"])
    for i in range(n):
        k = f"c{i:03d}"
        yield k, {s: z[k + "_" + s] for s in ("kv", "u0", "dt", "t", "u1", "deg", "ghost", "edt", "diag", "adm",
                                               "imexdt")}


IMEX_NAMES = ["gresho_m0p1", "gresho_m0p01", "bubble", "sod_reflect"]


def imex_case(name):
    z = load("imex_cases.npz")
    return {k[len(name) + 1:]: z[k] for k in z.files if k.startswith(name + "_")}


def state_rel_err(a, b):
    """max |a - b| over a state (4, ny, nx), relative per field family:
    density by max|rho|, both momentum components by the larger of max|mx|,
    max|my|, energy by max|E| (a momentum component that is identically
    zero up to rounding is thus measured against the flow's momentum)."""
    a = np.asarray(a)
    b = np.asarray(b)
    d = np.abs(a - b).reshape(4, -1).max(axis=1)
    s = np.abs(b).reshape(4, -1).max(axis=1)
    sm = max(s[1], s[2])
    scales = np.array([s[0], sm, sm, s[3]])
    scales[scales == 0] = 1.0
    return float((d / scales).max())
