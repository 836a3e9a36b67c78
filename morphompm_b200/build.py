"""Build the sm_100a shared library ``morphompm_b200/_lib/libmorphompm_b200.so``
in-tree with nvcc (no torch extension machinery: the library exports a plain C
ABI, declared in ``include/morphompm_b200.h``), and its bounds-checked twin
``libmorphompm_b200_checked.so`` (the same sources with MPM_CHECK_BOUNDS).
Setting MORPHOMPM_CHECKED=1 makes the package load the checked library.

    python -m morphompm_b200.build [--force] [--verbose] [--checked]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(OUT_DIR, "libmorphompm_b200.so")
# the same sources with every kernel index checked (MPM_CHECK_BOUNDS)
LIB_CHECKED = os.path.join(OUT_DIR, "libmorphompm_b200_checked.so")
SOURCES = ["capi.cu"]
HEADERS = ["mpm_common.cuh", "constitutive.cuh", "sort.cuh", "mpm_kernels.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _inputs():
    files = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    files.append(os.path.join(ROOT, "include", "morphompm_b200.h"))
    return files


def up_to_date(checked: bool = False) -> bool:
    lib = LIB_CHECKED if checked else LIB
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def build(force: bool = False, verbose: bool = False, extra=None, checked: bool = False) -> str:
    """Build the release library, or with checked=True the bounds-checked one."""
    lib = LIB_CHECKED if checked else LIB
    if not force and up_to_date(checked):
        return lib
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = lib + ".tmp"
    flags = list(extra or []) + (["-DMPM_CHECK_BOUNDS"] if checked else [])
    cmd = [_nvcc(), *NVCC_FLAGS, *flags, "-o", tmp] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed building {os.path.basename(lib)}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    os.replace(tmp, lib)
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/spill usage")
    ap.add_argument("--checked", action="store_true", help="the bounds-checked library")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_v else None
    print(build(force=a.force or a.ptxas_v, verbose=a.verbose or a.ptxas_v, extra=extra, checked=a.checked))


if __name__ == "__main__":
    main()
