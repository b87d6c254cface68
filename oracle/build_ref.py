"""Builds oracle/_ref/libref.so: the reference's own code behind the C APIs of oracle/ref_harness.cu
(the editors, GPUBaseDAG item codecs, DAGUtils::get_value, Path) and oracle/ref_v3_harness.cu (the
reference's host DAG MyGPUHashDAG<EMemoryType::CPU> and its writeTo / readFrom file format).

Test infrastructure (a second checker beside the oracle). The reference sources are compiled where
they lie (REFERENCE_SRC, default /root/reference/src); nothing is copied. Libraries the reference's
sources include but this machine lacks are replaced by the minimal stand-ins in oracle/ref_shim
(gsl-lite's span/narrow, TBB's parallel_for_each, and memory_host.cu for the reference's memory.cu);
nlohmann/json, which stats.h includes, is taken from the copy that ships inside an installed Python
package when one exists. cub_scan.cu uses thrust::raw_pointer_cast without including its header, so
it is compiled with thrust/memory.h included first. The output stays in oracle/_ref (git-ignored; it
travels with the repository snapshot).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIB = os.path.join(OUT_DIR, "libref.so")
SHIM = os.path.join(HERE, "ref_shim")
REFERENCE_SRC = os.environ.get("REFERENCE_SRC", "/root/reference/src")

# (source, extra flags); harness and shim paths are relative to oracle/, reference paths to REFERENCE_SRC
OWN_SOURCES = ["ref_harness.cu", "ref_v3_harness.cu", os.path.join("ref_shim", "memory_host.cu")]
REFERENCE_SOURCES = [
    ("dags/my_gpu_dags/my_gpu_hash_dag/my_gpu_hash_dag.cu", []),
    ("dags/my_gpu_dags/my_gpu_hash_dag/hash_tables/gpu_hash_table_base.cu", []),
    ("dags/my_gpu_dags/my_gpu_hash_dag/hash_tables/compact_acceleration_hash_table.cu", []),
    ("dags/my_gpu_dags/my_gpu_hash_dag/hash_tables/dynamic_slab_alloc.cu", []),
    ("dags/my_gpu_dags/cub/cub_scan.cu", ["-include", "thrust/memory.h"]),
    ("dags/my_gpu_dags/cub/cub_radix_sort.cu", []),
    ("dags/my_gpu_dags/cub/cub_select.cu", []),
]


def _json_include():
    for base in {sys.prefix, os.path.dirname(os.path.dirname(os.__file__))}:
        for hit in glob.glob(os.path.join(base, "**", "nlohmann", "json.hpp"), recursive=True):
            return os.path.dirname(os.path.dirname(hit))
    return None


def available() -> bool:
    return os.path.isdir(REFERENCE_SRC)


def _sources():
    own = [(os.path.join(HERE, s), []) for s in OWN_SOURCES]
    ref = [(os.path.join(REFERENCE_SRC, s), f) for s, f in REFERENCE_SOURCES]
    return own + ref


def build(force: bool = False) -> str | None:
    """Returns the library path, or None when the reference sources are not on this machine."""
    if not available():
        return LIB if os.path.exists(LIB) else None
    sources = _sources()
    deps = [s for s, _ in sources] + glob.glob(os.path.join(SHIM, "**", "*"), recursive=True) + [os.path.abspath(__file__)]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(p) for p in deps):
        return LIB
    inc = _json_include()
    if inc is None:
        raise RuntimeError("nlohmann/json.hpp not found: the reference headers cannot be compiled here")
    os.makedirs(OBJ_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    common = ["-std=c++20", "-O2", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math", "-fmad=false",
              "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a", "-I", SHIM, "-I", REFERENCE_SRC,
              "-I", inc, "-diag-suppress", "20011,20012,20013,20014,20015,177,550,2361"]

    def compile_one(item):
        src, extra = item
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        subprocess.check_call([nvcc] + common + extra + ["-c", src, "-o", obj])
        return obj

    with cf.ThreadPoolExecutor(max_workers=len(sources)) as ex:
        objs = list(ex.map(compile_one, sources))
    subprocess.check_call([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a"] + objs + ["-o", LIB + ".tmp"])
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
