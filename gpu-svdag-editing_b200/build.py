"""Builds libsvdag.so in-tree for sm_100a with nvcc (no JIT cache, no torch extension machinery)."""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsvdag.so")
SOURCES = ["svdag_ctx.cu", "svdag_tables.cu", "svdag_edit.cu", "svdag_scene.cu", "svdag_server.cu", "svdag_trace.cu", "svdag_tune.cu", "svdag_replay.cu", "svdag_io.cu", "svdag_v3.cu", "svdag_alt_tables.cu"]
HEADERS = ["svdag_device.cuh", "svdag_edit.cuh", "svdag_scene.cuh", "svdag_host.hpp", "svdag_hash.h", "svdag_alt_tables.cuh", "svdag_serve_geometry.h", "svdag_snapshot.h", "svdag_subtree.h"]
NVCC = os.environ.get("NVCC", "nvcc")

# -fmad=false: the editors' float predicates decide the DAG structure and the tracer's decide the
# hits; no multiply-add may be contracted so that both are bit-exact against the uncontracted oracle.
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
]


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def _compile(src: str, extra) -> str:
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(HERE, "..", "include", "svdag.h")]
    if os.path.exists(obj) and os.path.getmtime(obj) >= _newest(deps):
        return obj
    cmd = [NVCC, *NVCC_FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj + ".tmp"]
    subprocess.check_call(cmd)
    os.replace(obj + ".tmp", obj)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    if force:
        for f in os.listdir(BUILD):
            if f.endswith(".o"):
                os.remove(os.path.join(BUILD, f))
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), SOURCES))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        subprocess.check_call([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB + ".tmp",
                               *objs, "-lcudart"])
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build())
