"""Builds libecg.so (the CUDA hot path + C ABI) in-tree for sm_100a.

    python -m amrex_euler_allmach_explicit_imex_b200.build [--force] [-v]

Objects go to <package>/_build/, the library to <package>/libecg.so.  nvcc
cross-compiles without a GPU.  Per-file flags: the stencil kernels are built
twice, once without FMA contraction (bit-identical arithmetic mode) and once
with it (default fast mode).
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libecg.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O3",
          "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

# translation unit -> extra flags
SOURCES = {
    "stencil_exact.cu": ["-fmad=false"],
    "stencil_fast.cu": ["-fmad=true"],
    "imex_exact.cu": ["-fmad=false"],
    "imex_fast.cu": ["-fmad=true"],
    "gmres.cu": ["-fmad=true"],
    "capi.cu": [],
    "imex.cu": [],
    "batched.cu": ["-fmad=true"],
    "adjoint.cu": ["-fmad=true"],
    "noalloc.cu": [],
    "hoststage.cu": [],
    "peak.cu": [],
    "output.cu": ["-fmad=false"],
    "paper.cu": ["-fmad=false"],
}


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def _headers_mtime():
    files = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    files += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(f) for f in files), default=0.0)


def _compile(src, flags, force, verbose):
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    newest = max(os.path.getmtime(path), _headers_mtime(), os.path.getmtime(__file__))
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj, None
    cmd = [nvcc()] + ARCH + COMMON + flags + ["-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{src}:\n{r.stdout}\n{r.stderr}"
    return obj, None


def build(force=False, verbose=False):
    """Compiles every CUDA translation unit for sm_100a and links libecg.so."""
    os.makedirs(BUILD, exist_ok=True)
    present = {s: f for s, f in SOURCES.items() if os.path.exists(os.path.join(CSRC, s))}
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda kv: _compile(kv[0], kv[1], force, verbose), present.items()))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    objs = [o for o, _ in results]
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        tmp = LIB + ".tmp"
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    sys.exit(main())
