"""Builds oracle/_ref/libref.so: the reference's own host-callable code (editors, GPUBaseDAG item
codecs, DAGUtils::get_value, Path) behind the C API of oracle/ref_harness.cu.

Test infrastructure (a second checker beside the oracle). The reference sources are compiled where
they lie (REFERENCE_SRC, default /root/reference/src); nothing is copied. Two external libraries the
reference's headers include are absent from this machine and are replaced by the minimal stand-ins
in oracle/ref_shim (gsl-lite's span/narrow, TBB's parallel_for_each); nlohmann/json, which stats.h
includes, is taken from the copy that ships inside an installed Python package when one exists.
The output stays in oracle/_ref (git-ignored; it travels with the repository snapshot).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libref.so")
SRC = os.path.join(HERE, "ref_harness.cu")
SHIM = os.path.join(HERE, "ref_shim")
REFERENCE_SRC = os.environ.get("REFERENCE_SRC", "/root/reference/src")


def _json_include():
    for base in {sys.prefix, os.path.dirname(os.path.dirname(os.__file__))}:
        for hit in glob.glob(os.path.join(base, "**", "nlohmann", "json.hpp"), recursive=True):
            return os.path.dirname(os.path.dirname(hit))
    return None


def available() -> bool:
    return os.path.isdir(REFERENCE_SRC)


def build(force: bool = False) -> str | None:
    """Returns the library path, or None when the reference sources are not on this machine."""
    if not available():
        return LIB if os.path.exists(LIB) else None
    deps = [SRC] + glob.glob(os.path.join(SHIM, "**", "*"), recursive=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(p) for p in deps):
        return LIB
    inc = _json_include()
    if inc is None:
        raise RuntimeError("nlohmann/json.hpp not found: the reference headers cannot be compiled here")
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [os.environ.get("NVCC", "nvcc"), "-std=c++20", "-O2", "-shared", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
           "-fmad=false", "-gencode", "arch=compute_100a,code=sm_100a", "-I", SHIM, "-I", REFERENCE_SRC, "-I", inc,
           "-diag-suppress", "20012,20013,20014,20015,177,550,2361", SRC, "-o", LIB + ".tmp"]
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
