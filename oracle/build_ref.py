"""Compile the reference's C++ forward solver (header-only, read in place from
the reference tree) behind the C ABI of growth_ref.cpp into oracle/_ref/.

    python oracle/build_ref.py [--ref /path/to/reference]

Test infrastructure: the library is a checker and a timed CPU baseline, never
part of the product.  Without the reference tree nothing is built.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref", "libgrowth_ref.so")
# Where this recipe reads the reference sources in the build container; the
# MORPHOMPM_REF environment variable or --ref points it elsewhere.
REF_MOUNT = "/root/reference"


def ref_root() -> str:
    """Root of the reference project: MORPHOMPM_REF, else the build container's mount."""
    return os.environ.get("MORPHOMPM_REF") or REF_MOUNT


def build(ref_root: str, quiet: bool = False) -> str | None:
    inc = os.path.join(ref_root, "include")
    if not os.path.isfile(os.path.join(inc, "morphompm", "growth_solver.h")):
        if not quiet:
            print("reference tree not found; oracle/_ref not built", file=sys.stderr)
        return None
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-mavx2", "-mfma", "-fPIC", "-shared", "-I", inc,
           os.path.join(HERE, "growth_ref.cpp"), "-o", OUT]
    subprocess.run(cmd, check=True)
    return OUT


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference root (default: MORPHOMPM_REF, else the build mount)")
    a = ap.parse_args()
    out = build(a.ref or ref_root())
    if out:
        print(out)


if __name__ == "__main__":
    main()
