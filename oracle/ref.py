"""ctypes binding of oracle/_ref/libref.so: the reference's own editors, item codecs and
DAGUtils::get_value (oracle/ref_harness.cu), and its host DAG with the writeTo / readFrom file
format (oracle/ref_v3_harness.cu), built by oracle/build_ref.py.

TEST INFRASTRUCTURE ONLY: the tests use it to check the oracle (and, on a GPU, the CUDA library's
exported DAG) against reference code. `lib()` returns None where the library is neither built nor
buildable (no reference sources on this machine).
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libref.so")

_lib = None
_tried = False


def _recipe():
    spec = importlib.util.spec_from_file_location("build_ref", os.path.join(HERE, "build_ref.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def lib():
    global _lib, _tried
    if _lib is not None or _tried:
        return _lib
    _tried = True
    path = _recipe().build()
    if not path or not os.path.exists(path):
        return None
    L = C.CDLL(path)
    P = C.c_void_p
    L.ref_dag_create.restype = P
    L.ref_dag_create.argtypes = [C.c_uint32, P, C.c_uint64]
    L.ref_dag_destroy.argtypes = [P]
    L.ref_dag_destroy.restype = None
    L.ref_get_values.argtypes = [P, P, C.c_uint64, P]
    L.ref_edit_values.argtypes = [P, P, P, C.c_uint64, P]
    L.ref_should_edit.argtypes = [P, P, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32)]
    L.ref_should_edit_many.argtypes = [P, P, P, P, P, C.c_uint64, P, P]
    L.ref_build_leaf.restype = C.c_uint32
    L.ref_build_leaf.argtypes = [P, P]
    L.ref_leaf_size.restype = C.c_uint32
    L.ref_leaf_size.argtypes = [P]
    L.ref_leaf_material.argtypes = [P, C.c_uint32, C.POINTER(C.c_uint32)]
    for f in ("ref_encode_node_header", "ref_encode_full_node_header"):
        getattr(L, f).restype = C.c_uint32
        getattr(L, f).argtypes = [C.c_uint32, C.c_uint32]
    L.ref_header_fully_filled.argtypes = [C.c_uint32, C.POINTER(C.c_uint32)]
    L.ref_v3_levels.restype = C.c_uint32
    L.ref_v3_levels.argtypes = []
    L.ref_v3_write.argtypes = [P, P, P, C.c_char_p]
    L.ref_v3_open.restype = P
    L.ref_v3_open.argtypes = [C.c_char_p]
    L.ref_v3_close.restype = None
    L.ref_v3_close.argtypes = [P]
    L.ref_v3_root.restype = C.c_uint32
    L.ref_v3_root.argtypes = [P]
    L.ref_v3_items.argtypes = [P, P, C.c_uint64, P, P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.ref_v3_get_values.argtypes = [P, P, C.c_uint64, P]
    _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class RefDag:
    """A DAG given as items of 10 words with children as item indices (row 0 = root), read by the
    reference's own code."""

    def __init__(self, levels: int, items: np.ndarray):
        self.items = np.ascontiguousarray(items, dtype=np.uint32).reshape(-1, 10)
        self.levels = levels
        self.h = lib().ref_dag_create(levels, _p(self.items), len(self.items))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ref_dag_destroy(self.h)
            self.h = None

    def get_values(self, xyz: np.ndarray) -> np.ndarray:
        xyz = np.ascontiguousarray(xyz, dtype=np.uint32).reshape(-1, 3)
        out = np.empty(len(xyz), dtype=np.uint32)
        lib().ref_get_values(self.h, _p(xyz), len(xyz), _p(out))
        return out

    def edit_values(self, edit, xyz: np.ndarray) -> np.ndarray:
        """Values of the voxels after `edit` (an svdag_edit-layout ctypes structure), decided by
        the reference's editor over this DAG as it is before the edit."""
        xyz = np.ascontiguousarray(xyz, dtype=np.uint32).reshape(-1, 3)
        out = np.empty(len(xyz), dtype=np.uint32)
        if lib().ref_edit_values(self.h, C.byref(edit), _p(xyz), len(xyz), _p(out)) != 0:
            raise ValueError("the reference has no editor for this tool")
        return out


def items_from_dumps(levels: int, root: int, dumps) -> np.ndarray:
    """Rewrites per-level dumps (handles, words) of a DAG, e.g. the CUDA library's export_level,
    into the item array RefDag takes: the items reachable from `root`, children as row indices."""
    index = [dict(zip(h.tolist(), range(len(h)))) for h, _ in dumps]
    rows, where = [], {}
    frontier = [root]
    for level in range(levels - 1):
        nxt = []
        for h in frontier:
            if (level, h) in where:
                continue
            where[(level, h)] = len(rows)
            w = dumps[level][1][index[level][h]].copy()
            rows.append(w)
            if level < levels - 2:
                k = bin(int(w[0]) & 0xFF).count("1")
                nxt.extend(int(c) for c in w[1:1 + k])
        frontier = nxt
    out = np.array(rows, dtype=np.uint32).reshape(-1, 10)
    for level in range(levels - 2):
        for (lv, h), r in where.items():
            if lv != level:
                continue
            k = bin(int(out[r, 0]) & 0xFF).count("1")
            out[r, 1:1 + k] = [where[(level + 1, int(c))] for c in out[r, 1:1 + k]]
    return out


def v3_levels() -> int:
    """The scene depth the reference's DAG was compiled with (SCENE_DEPTH)."""
    return int(lib().ref_v3_levels())


def v3_write(words: np.ndarray, level_words: np.ndarray, level_items: np.ndarray, path: str):
    """Builds the reference's host DAG from an item snapshot of v3_levels() levels and writes it
    with MyGPUHashDAG::writeTo. Needs a CUDA driver (the reference's host arrays are copied with
    cudaMemcpy)."""
    w = np.ascontiguousarray(words, dtype=np.uint32)
    lw = np.ascontiguousarray(level_words, dtype=np.uint64)
    li = np.ascontiguousarray(level_items, dtype=np.uint64)
    if lib().ref_v3_write(_p(w) if len(w) else None, _p(lw), _p(li), os.fsencode(path)) != 0:
        raise ValueError("the snapshot does not parse")


class RefV3Dag:
    """A version-3 DAG file loaded by the reference's MyGPUHashDAG::readFrom (host memory; needs a
    CUDA driver, like v3_write)."""

    def __init__(self, path: str):
        self.h = lib().ref_v3_open(os.fsencode(path))

    def close(self):
        if self.h:
            lib().ref_v3_close(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def root(self) -> int:
        return int(lib().ref_v3_root(self.h))

    def items(self):
        """(words, level_words, level_items, found): the reachable items as a snapshot read through
        the reference's accessors, and how many of them its find locates at their own handle."""
        nl = v3_levels() - 1
        lw, li = np.zeros(nl, np.uint64), np.zeros(nl, np.uint64)
        total, found = C.c_uint64(), C.c_uint64()
        lib().ref_v3_items(self.h, None, 0, _p(lw), _p(li), C.byref(total), C.byref(found))
        words = np.zeros(max(total.value, 1), np.uint32)
        assert lib().ref_v3_items(self.h, _p(words), len(words), _p(lw), _p(li), C.byref(total), C.byref(found)) == 0
        return words[: total.value], lw, li, found.value

    def get_values(self, xyz: np.ndarray) -> np.ndarray:
        xyz = np.ascontiguousarray(xyz, dtype=np.uint32).reshape(-1, 3)
        out = np.empty(len(xyz), dtype=np.uint32)
        lib().ref_v3_get_values(self.h, _p(xyz), len(xyz), _p(out))
        return out
