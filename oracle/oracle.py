"""ctypes binding of the CPU oracle (oracle/svdag_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the checker and by
bench.py's cpu_baseline / reference leg. The product never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
SOURCES = [os.path.join(HERE, "svdag_oracle.cpp")]
CXXFLAGS = ["-std=c++20", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-Wall"]

MAX_LEVELS = 17
MAX_ITEM_WORDS = 10


def build(force: bool = False) -> str:
    """Compiles the oracle with g++ (no contraction, no fast-math)."""
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    newest = max(os.path.getmtime(p) for p in SOURCES + [os.path.join(HERE, "svdag_oracle.h")])
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < newest:
        tmp = LIB_PATH + ".tmp"
        subprocess.check_call(["g++", *CXXFLAGS, "-o", tmp, *SOURCES, "-lpthread"])
        os.replace(tmp, LIB_PATH)
    return LIB_PATH


class TerrainParams(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("octaves", C.c_uint32), ("num_materials", C.c_uint32),
                ("min_height_pct", C.c_uint32), ("max_height_pct", C.c_uint32),
                ("num_structures", C.c_uint32), ("structure_seed", C.c_uint32), ("tile_level", C.c_uint32)]


class Edit(C.Structure):
    _fields_ = [("tool", C.c_uint32), ("material", C.c_uint32), ("center", C.c_float * 3),
                ("radius", C.c_float), ("src", C.c_float * 3), ("dst", C.c_float * 3),
                ("noise_seed", C.c_uint32), ("noise_cell_log2", C.c_uint32)]


class EditStats(C.Structure):
    _fields_ = [("svo_nodes", C.c_uint64 * MAX_LEVELS), ("old_items_read", C.c_uint64),
                ("unique_items", C.c_uint64), ("new_items", C.c_uint64), ("edited_voxels", C.c_uint64),
                ("root_before", C.c_uint32), ("root_after", C.c_uint32), ("status", C.c_uint32),
                ("reserved", C.c_uint32)]


class TraceParams(C.Structure):
    _fields_ = [("camera", C.c_double * 3), ("ray_min", C.c_double * 3), ("ray_ddx", C.c_double * 3),
                ("ray_ddy", C.c_double * 3), ("width", C.c_uint32), ("height", C.c_uint32)]


class ShadeParams(C.Structure):
    _fields_ = [("material_srgb8", C.c_uint32 * 16), ("sun_direction", C.c_float * 3), ("shadow_bias", C.c_float),
                ("ao_ray_length", C.c_float), ("sun_brightness", C.c_float), ("fog_density", C.c_float),
                ("ao_samples", C.c_uint32), ("flags", C.c_uint32), ("pad", C.c_uint32), ("random_seed", C.c_uint64)]


HIT_DTYPE = np.dtype([("path", "<u4", (3,)), ("material", "u1"), ("pad", "u1", (3,)),
                      ("position", "<f4", (3,)), ("normal", "<f4", (3,)), ("dpdu", "<f4", (3,)),
                      ("dpdv", "<f4", (3,)), ("color", "<u4")])
assert HIT_DTYPE.itemsize == 68


class Canon(C.Structure):
    _fields_ = [("unique_per_level", C.c_uint64 * MAX_LEVELS), ("digest_per_level", C.c_uint64 * MAX_LEVELS),
                ("root_digest", C.c_uint64), ("voxel_count_lo", C.c_uint64), ("voxel_count_hi", C.c_uint64)]

    def as_dict(self, levels: int) -> dict:
        return {"unique": [int(self.unique_per_level[i]) for i in range(levels - 1)],
                "digest": [int(self.digest_per_level[i]) for i in range(levels - 1)],
                "root": int(self.root_digest),
                "voxels": int(self.voxel_count_lo) | (int(self.voxel_count_hi) << 64)}


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(build())
        P = C.c_void_p
        L.oracle_create.restype = P
        L.oracle_create.argtypes = [C.c_uint32]
        L.oracle_destroy.argtypes = [P]
        L.oracle_root.restype = C.c_uint32
        L.oracle_root.argtypes = [P]
        L.oracle_levels.restype = C.c_uint32
        L.oracle_levels.argtypes = [P]
        L.oracle_is_empty.argtypes = [P]
        L.oracle_build_terrain.argtypes = [P, C.POINTER(TerrainParams)]
        L.oracle_build_box.argtypes = [P, C.c_float, C.c_float, C.c_uint32]
        L.oracle_edit.argtypes = [P, C.POINTER(Edit), C.POINTER(EditStats)]
        for f in ("oracle_undo", "oracle_redo", "oracle_gc"):
            getattr(L, f).argtypes = [P]
        for f in ("oracle_undo_count", "oracle_redo_count"):
            getattr(L, f).argtypes = [P]
            getattr(L, f).restype = C.c_uint32
        L.oracle_sample_voxels.argtypes = [P, P, C.c_uint64, P]
        L.oracle_export_items.argtypes = [P, P, C.c_uint64, C.POINTER(C.c_uint64)]
        L.oracle_should_edit_many.argtypes = [C.c_void_p, P, P, P, P, C.c_uint64, P, P]
        L.oracle_trace.argtypes = [P, C.POINTER(TraceParams), P, C.c_int]
        L.oracle_shade.argtypes = [P, C.POINTER(TraceParams), C.POINTER(ShadeParams), P, P, P, P, C.c_int]
        L.oracle_sincos.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.oracle_sincos.restype = None
        L.oracle_trace_counts.argtypes = [P, C.POINTER(TraceParams), C.POINTER(C.c_uint64),
                                          C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.oracle_canonicalize.argtypes = [P, C.POINTER(Canon)]
        L.oracle_canonicalize_dump.argtypes = [C.c_uint32, C.c_uint32, P, P, P, C.POINTER(Canon)]
        L.oracle_canonicalize_dump_at.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, P, P, P, C.POINTER(Canon)]
        L.oracle_canonicalize_at.argtypes = [P, C.c_uint32, C.c_uint32, C.POINTER(Canon)]
        L.oracle_build_scene_subtree.argtypes = [P, C.POINTER(TerrainParams), C.c_uint32, P, C.POINTER(C.c_uint32)]
        L.oracle_scene_voxels.argtypes = [C.POINTER(TerrainParams), C.c_uint32, P, C.c_uint64, P]
        L.oracle_build_scene_region.argtypes = [P, C.POINTER(TerrainParams), P, P]
        L.oracle_node_at.restype = C.c_uint32
        L.oracle_node_at.argtypes = [P, C.c_uint32, P]
        L.oracle_encode_node_header.restype = C.c_uint32
        L.oracle_encode_node_header.argtypes = [C.c_uint32, C.c_uint32]
        L.oracle_header_child_mask.restype = C.c_uint32
        L.oracle_header_child_mask.argtypes = [C.c_uint32]
        L.oracle_header_user_payload.restype = C.c_uint32
        L.oracle_header_user_payload.argtypes = [C.c_uint32]
        L.oracle_build_leaf.restype = C.c_uint32
        L.oracle_build_leaf.argtypes = [C.c_uint64, P, P]
        L.oracle_leaf_size.restype = C.c_uint32
        L.oracle_leaf_size.argtypes = [P]
        L.oracle_leaf_material.argtypes = [P, C.c_uint32, C.POINTER(C.c_uint32)]
        L.oracle_terrain_height.restype = C.c_uint32
        L.oracle_terrain_height.argtypes = [C.POINTER(TerrainParams), C.c_uint32, C.c_uint32, C.c_uint32]
        L.oracle_noise_material.restype = C.c_uint32
        L.oracle_noise_material.argtypes = [C.c_uint32] * 5
        L.oracle_should_edit.argtypes = [C.POINTER(Edit), P, C.c_uint32, C.c_uint32, C.c_uint32,
                                         C.POINTER(C.c_uint32)]
        L.oracle_camera_params.argtypes = [P, P, C.c_double, C.c_uint32, C.c_uint32, C.POINTER(TraceParams)]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class OracleDag:
    """A DAG held by the CPU oracle."""

    def __init__(self, levels: int):
        self.levels = levels
        self.h = lib().oracle_create(levels)
        if not self.h:
            raise ValueError(f"unsupported depth {levels}")

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().oracle_destroy(self.h)
            except Exception:  # interpreter shutdown
                pass
            self.h = None

    @property
    def root(self) -> int:
        return lib().oracle_root(self.h)

    def build_terrain(self, params: TerrainParams):
        r = lib().oracle_build_terrain(self.h, C.byref(params))
        if r:
            raise RuntimeError(f"oracle_build_terrain -> {r}")

    def build_scene_subtree(self, params: TerrainParams, level: int, path) -> int:
        """Builds only the subtree of scene node (level, path); returns its handle at `level`."""
        p = np.ascontiguousarray(path, dtype=np.uint32)
        h = C.c_uint32()
        r = lib().oracle_build_scene_subtree(self.h, C.byref(params), level, _ptr(p), C.byref(h))
        if r:
            raise RuntimeError(f"oracle_build_scene_subtree -> {r}")
        return h.value

    def build_scene_region(self, params: TerrainParams, lo, hi):
        """Builds the scene with every voxel outside the box [lo, hi) empty."""
        a = np.ascontiguousarray(lo, dtype=np.int64)
        b = np.ascontiguousarray(hi, dtype=np.int64)
        r = lib().oracle_build_scene_region(self.h, C.byref(params), _ptr(a), _ptr(b))
        if r:
            raise RuntimeError(f"oracle_build_scene_region -> {r}")

    def node_at(self, level: int, path):
        """Handle of node (level, path), or None where the DAG is empty."""
        p = np.ascontiguousarray(path, dtype=np.uint32)
        h = lib().oracle_node_at(self.h, level, _ptr(p))
        return None if h == 0xFFFFFFFF else h

    def canon_at(self, level: int, handle: int) -> dict:
        c = Canon()
        lib().oracle_canonicalize_at(self.h, level, handle, C.byref(c))
        return c.as_dict(self.levels)

    def build_box(self, bmin: float, bmax: float, material: int):
        lib().oracle_build_box(self.h, bmin, bmax, material)

    def edit(self, e: Edit) -> EditStats:
        st = EditStats()
        r = lib().oracle_edit(self.h, C.byref(e), C.byref(st))
        if r:
            raise RuntimeError(f"oracle_edit -> {r}")
        return st

    def undo(self):
        lib().oracle_undo(self.h)

    def redo(self):
        lib().oracle_redo(self.h)

    def gc(self):
        lib().oracle_gc(self.h)

    def undo_count(self) -> int:
        return lib().oracle_undo_count(self.h)

    def redo_count(self) -> int:
        return lib().oracle_redo_count(self.h)

    def export_items(self) -> np.ndarray:
        """Items reachable from the root, (n, 10) uint32, children as row indices, row 0 = root."""
        n = C.c_uint64()
        lib().oracle_export_items(self.h, None, 0, C.byref(n))
        out = np.zeros((n.value, 10), dtype=np.uint32)
        if n.value:
            lib().oracle_export_items(self.h, _ptr(out), n.value, C.byref(n))
        return out

    def sample(self, xyz: np.ndarray) -> np.ndarray:
        xyz = np.ascontiguousarray(xyz, dtype=np.uint32).reshape(-1, 3)
        out = np.empty(len(xyz), dtype=np.uint32)
        lib().oracle_sample_voxels(self.h, _ptr(xyz), len(xyz), _ptr(out))
        return out

    def trace(self, params: TraceParams, threads: int = 1) -> np.ndarray:
        out = np.zeros(params.width * params.height, dtype=HIT_DTYPE)
        lib().oracle_trace(self.h, C.byref(params), _ptr(out), threads)
        return out

    def shade(self, params: TraceParams, shade: ShadeParams, hits: np.ndarray, threads: int = 8):
        """(hits with diffuse colours, rgba uint32, sun float32, ao float32) of a traced hit buffer."""
        hits = hits.copy()
        n = params.width * params.height
        rgba, sun, ao = np.zeros(n, np.uint32), np.zeros(n, np.float32), np.zeros(n, np.float32)
        lib().oracle_shade(self.h, C.byref(params), C.byref(shade), _ptr(hits), _ptr(rgba), _ptr(sun), _ptr(ao), threads)
        return hits, rgba, sun, ao

    def trace_counts(self, params: TraceParams):
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        lib().oracle_trace_counts(self.h, C.byref(params), C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def canon(self) -> dict:
        c = Canon()
        lib().oracle_canonicalize(self.h, C.byref(c))
        return c.as_dict(self.levels)


def scene_voxels(params: TerrainParams, levels: int, xyz: np.ndarray) -> np.ndarray:
    """Voxels of the scene straight from its definition (no DAG)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.uint32).reshape(-1, 3)
    out = np.empty(len(xyz), dtype=np.uint32)
    lib().oracle_scene_voxels(C.byref(params), levels, _ptr(xyz), len(xyz), _ptr(out))
    return out


def canonicalize_dump(levels: int, root: int, dumps, level: int = 0) -> dict:
    """dumps[l] = (handles uint32[n], words uint32[n, 10]) for every level 0..levels-2; `root` is an
    item of `level`."""
    n = levels - 1
    hs = [np.ascontiguousarray(d[0], dtype=np.uint32) for d in dumps]
    ws = [np.ascontiguousarray(d[1], dtype=np.uint32) for d in dumps]
    hp = (C.c_void_p * n)(*[h.ctypes.data for h in hs])
    wp = (C.c_void_p * n)(*[w.ctypes.data for w in ws])
    counts = np.array([len(h) for h in hs], dtype=np.uint64)
    c = Canon()
    r = lib().oracle_canonicalize_dump_at(levels, level, root, hp, wp, _ptr(counts), C.byref(c))
    if r:
        raise RuntimeError("dump references a handle that is not in the dump")
    return c.as_dict(levels)


def camera_params(position, target, fov_degrees: float, width: int, height: int) -> TraceParams:
    p = TraceParams()
    pos = np.array(position, dtype=np.float64)
    tgt = np.array(target, dtype=np.float64)
    lib().oracle_camera_params(_ptr(pos), _ptr(tgt), fov_degrees, width, height, C.byref(p))
    return p
