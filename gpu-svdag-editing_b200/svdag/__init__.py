"""Python host binding of libsvdag (C ABI declared in include/svdag.h).

The names mirror the reference's EDag::MyGpuDag interface (mathijs727/GPU-SVDAG-Editing):
``MyGPUHashDAG`` (my_gpu_hash_dag.h), the tool classes of my_gpu_dag_editors.h, ``editMyHashDag``
(my_gpu_hash_dag_edits.h:12-13), ``MyGPUHashDAGUndoRedo`` (my_gpu_base_dag.h:16-82) and
``DAGTracer.resolve_paths`` (dag_tracer.h:33). Every call goes through the CUDA library; there is no
CPU path: importing this module on a machine where libsvdag.so is missing raises, and creating a
context without an sm_100 device raises ``SvdagError(SVDAG_ERR_NO_DEVICE)``.

Device buffers and streams are plain CUDA pointers; torch tensors are accepted for convenience
(``.data_ptr()`` / ``torch.cuda.Stream.cuda_stream``).
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG_ROOT, "libsvdag.so")

MAX_LEVELS = 17
V3_GPU_MANAGED, V3_GPU_MALLOC, V3_GPU_ASYNC, V3_CPU = 0, 1, 2, 3  # EMemoryType values of a v3 file, memory.h:17-23
MAX_ITEM_WORDS = 10
NUM_SIZE_CLASSES = 9
NUM_MATERIALS = 16
INVALID_HANDLE = 0xFFFFFFFF
NO_MATERIAL = 0xFFFFFFFF

KIND_NODE, KIND_LEAF = 0, 1

TOOL_SPHERE_ADD, TOOL_SPHERE_REMOVE, TOOL_BOX_ADD, TOOL_BOX_REMOVE = 0, 1, 2, 3
TOOL_SPHERE_PAINT, TOOL_COPY, TOOL_BOX_PAINT_NOISE, TOOL_MOVE = 4, 5, 6, 7
TOOL_SPHERE_ERODE = 8

STATUS = {0: "SVDAG_OK", 1: "SVDAG_ERR_INVALID", 2: "SVDAG_ERR_OOM", 3: "SVDAG_ERR_TIMEOUT",
          4: "SVDAG_ERR_CORRUPT", 5: "SVDAG_ERR_CUDA", 6: "SVDAG_ERR_NO_DEVICE", 7: "SVDAG_ERR_UNSUPPORTED",
          8: "SVDAG_ERR_BUSY"}


class SvdagError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, status)}")


class Config(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("device", C.c_int32), ("pool_bytes", C.c_uint64),
                ("scratch_bytes", C.c_uint64), ("target_load_factor", C.c_uint32), ("probe_lanes", C.c_uint32),
                ("undo_depth", C.c_uint32), ("flags", C.c_uint32)]


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


class EditRecord(C.Structure):
    _fields_ = [("root_before", C.c_uint32), ("root_after", C.c_uint32), ("status", C.c_uint32),
                ("reserved", C.c_uint32), ("edited_voxels", C.c_uint64), ("new_items", C.c_uint64),
                ("unique_items", C.c_uint64), ("svo_items", C.c_uint64)]


class TraceParams(C.Structure):
    _fields_ = [("camera", C.c_double * 3), ("ray_min", C.c_double * 3), ("ray_ddx", C.c_double * 3),
                ("ray_ddy", C.c_double * 3), ("width", C.c_uint32), ("height", C.c_uint32)]


class ServerConfig(C.Structure):
    _fields_ = [("max_batch", C.c_uint32), ("max_inflight", C.c_uint32), ("memory_cap_bytes", C.c_uint64),
                ("frame", TraceParams), ("flags", C.c_uint32), ("reserved", C.c_uint32),
                ("gc_threshold_bytes", C.c_uint64)]


class ServerMemory(C.Structure):
    """svdag_server_memory: the serving loop's memory accounting and in-loop collections."""
    _fields_ = [("used_bytes", C.c_uint64), ("cap_bytes", C.c_uint64), ("gc_threshold_bytes", C.c_uint64),
                ("gc_runs", C.c_uint64), ("gc_freed_bytes", C.c_uint64), ("gc_seconds", C.c_double),
                ("rejected_edits", C.c_uint64), ("failed_edits", C.c_uint64), ("reuse_credit_bytes", C.c_uint64)]


class RequestResult(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("kind", C.c_uint32), ("status", C.c_uint32), ("root_after", C.c_uint32),
                ("launch", C.c_uint32), ("edited_voxels", C.c_uint64), ("submit_s", C.c_double),
                ("visible_s", C.c_double)]


class ReplayAction(C.Structure):
    """svdag_replay_action: one line of a reference replay file (replay.h)."""
    _fields_ = [("kind", C.c_uint32), ("edit", Edit), ("camera", C.c_float * 9)]


REPLAY_OTHER, REPLAY_EDIT, REPLAY_UNDO, REPLAY_REDO, REPLAY_END_FRAME = 0, 1, 2, 3, 4
REPLAY_CAMERA_LOCATION, REPLAY_CAMERA_ROTATION = 5, 6
RESULT_EDIT, RESULT_FRAME, RESULT_UNDO, RESULT_REDO = 0, 1, 2, 3

RESULT_DTYPE = np.dtype([("ticket", "<u8"), ("kind", "<u4"), ("status", "<u4"), ("root_after", "<u4"),
                         ("launch", "<u4"), ("edited_voxels", "<u8"), ("submit_s", "<f8"), ("visible_s", "<f8")])
assert RESULT_DTYPE.itemsize == C.sizeof(RequestResult) == 48

SERVE_PLAIN, SERVE_COPY_FRAMES, SERVE_FULL_FRAMES, SERVE_NO_GC = 1, 2, 4, 8


class ShadeParams(C.Structure):
    _fields_ = [("material_srgb8", C.c_uint32 * NUM_MATERIALS), ("sun_direction", C.c_float * 3),
                ("shadow_bias", C.c_float), ("ao_ray_length", C.c_float), ("sun_brightness", C.c_float),
                ("fog_density", C.c_float), ("ao_samples", C.c_uint32), ("flags", C.c_uint32), ("pad", C.c_uint32),
                ("random_seed", C.c_uint64)]


SHADE_SHADOWS, SHADE_AO = 1, 2
# Diffuse sRGB8 colour per material (0x00BBGGRR): stands in for the reference's material textures.
DEFAULT_PALETTE = (0x3C5A7A, 0x4A7F5B, 0x2E6B8C, 0x8C8C8C, 0x5E5E5E, 0x3B8FD4, 0x61A0A8, 0xD9D9D9,
                   0x2F2FB0, 0x2E9AE8, 0x3DB86A, 0xB06A2F, 0x8A3DB8, 0x6AD4E0, 0x1F4E79, 0xF0F0F0)


def shade_params(levels: int, shadows: bool = True, ao_samples: int = 0, ao_ray_length: float | None = None,
                 shadow_bias: float = 1.0, sun_brightness: float = 1.0, fog_density: float = 0.0, seed: int = 1,
                 palette=DEFAULT_PALETTE) -> ShadeParams:
    """Shading parameters with the reference engine's defaults (engine.h:212-214): shadow bias 1, AO
    ray length 2^(levels - 10), the sun towards normalize(0.3, 1, 0.5) (computed in double)."""
    sun = np.array([0.3, 1.0, 0.5])
    sun = sun / math.sqrt(float(np.dot(sun, sun)))
    p = ShadeParams()
    p.material_srgb8[:] = list(palette)
    p.sun_direction[:] = [float(np.float32(v)) for v in sun]
    p.shadow_bias = shadow_bias
    p.ao_ray_length = float(1 << max(levels - 10, 0)) if ao_ray_length is None else ao_ray_length
    p.sun_brightness = sun_brightness
    p.fog_density = fog_density
    p.ao_samples = ao_samples
    p.flags = (SHADE_SHADOWS if shadows else 0) | (SHADE_AO if ao_samples else 0)
    p.random_seed = seed
    return p


class Tuning(C.Structure):
    _fields_ = [("probe_lanes", C.c_uint32), ("load_factor", C.c_uint32), ("persistent_leaves", C.c_uint32),
                ("trials", C.c_uint32), ("table_ns_per_key", C.c_double), ("graph_us_small", C.c_double),
                ("persistent_us_small", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("root", C.c_uint32), ("pool_bytes", C.c_uint64),
                ("item_region_bytes", C.c_uint64), ("item_region_used_bytes", C.c_uint64),
                ("scratch_bytes", C.c_uint64), ("scratch_high_water_bytes", C.c_uint64),
                ("level_items", C.c_uint64 * MAX_LEVELS), ("level_buckets", C.c_uint64 * MAX_LEVELS),
                ("undo_count", C.c_uint32), ("redo_count", C.c_uint32), ("free_list_bytes", C.c_uint64),
                ("free_list_slabs", C.c_uint64), ("gc_freed_items", C.c_uint64), ("gc_freed_slabs", C.c_uint64),
                ("gc_live_items", C.c_uint64)]


class TableStats(C.Structure):
    _fields_ = [("items", C.c_uint64), ("buckets", C.c_uint64), ("overflow_slabs", C.c_uint64),
                ("bytes", C.c_uint64)]


# Tracer::SurfaceInteraction (tracer.h:95-110), 68 bytes.
HIT_DTYPE = np.dtype([("path", "<u4", (3,)), ("material", "u1"), ("pad", "u1", (3,)),
                      ("position", "<f4", (3,)), ("normal", "<f4", (3,)), ("dpdu", "<f4", (3,)),
                      ("dpdv", "<f4", (3,)), ("color", "<u4")])
assert HIT_DTYPE.itemsize == 68

_P = C.c_void_p
_U32, _U64 = C.c_uint32, C.c_uint64
_PROTOS = {
    "svdag_create": [C.POINTER(Config), C.POINTER(_P)],
    "svdag_destroy": [_P],
    "svdag_sync": [_P, _P],
    "svdag_status_string": [C.c_int],
    "svdag_abi_version": [],
    "svdag_build_terrain": [_P, C.POINTER(TerrainParams), _P],
    "svdag_scene_height": [C.POINTER(TerrainParams), _U32, _U32, _U32],
    "svdag_edit_apply": [_P, C.POINTER(Edit), _P],
    "svdag_edit_apply_many": [_P, C.POINTER(Edit), _U32, _P],
    "svdag_last_edit_stats": [_P, C.POINTER(EditStats), _P],
    "svdag_edit_records": [_P, C.POINTER(EditRecord), _U32, _P],
    "svdag_last_edit_phase_times": [_P, _P, _U32, C.POINTER(_U32), _P],
    "svdag_edit_sphere": [_P, C.c_float, C.c_float, C.c_float, C.c_float, _U32, C.c_int, _P],
    "svdag_edit_box": [_P, C.c_float, C.c_float, C.c_float, C.c_float, _U32, C.c_int, _P],
    "svdag_edit_paint": [_P, C.c_float, C.c_float, C.c_float, C.c_float, _U32, _P],
    "svdag_edit_paint_noise": [_P, C.c_float, C.c_float, C.c_float, C.c_float, _U32, _U32, _P],
    "svdag_edit_copy": [_P, _P, _P, _P, C.c_float, _P],
    "svdag_undo": [_P, _P],
    "svdag_redo": [_P, _P],
    "svdag_gc": [_P, _P],
    "svdag_gc_keep_history": [_P, _P],
    "svdag_get_root": [_P, C.POINTER(_U32), _P],
    "svdag_trace_primary": [_P, C.POINTER(TraceParams), _P, _P],
    "svdag_sample_voxels": [_P, _P, _U32, _P, _P],
    "svdag_level_table": [_P, _U32, C.POINTER(_P)],
    "svdag_table_create": [_P, _U32, _P, C.POINTER(_P)],
    "svdag_table_destroy": [_P],
    "svdag_table_add": [_P, _P, _P, _U32, _U64, _P, _U32, _P],
    "svdag_table_find": [_P, _P, _P, _U32, _U64, _P, _U32, _P],
    "svdag_table_find_or_add": [_P, _P, _P, _U32, _U64, _P, _U32, _P],
    "svdag_table_find_or_add_static": [_P, _P, _P, _U32, _U64, _P, _U32, _P],
    "svdag_table_read": [_P, _P, _U32, _P, _P],
    "svdag_table_get_stats": [_P, C.POINTER(TableStats), _P],
    "svdag_alt_table_create": [_P, _U32, _U32, _U32, _U64, C.POINTER(_P)],
    "svdag_alt_table_destroy": [_P],
    "svdag_alt_table_add": [_P, _P, _U32, _P, _U32, _P],
    "svdag_alt_table_find": [_P, _P, _U32, _P, _U32, _P],
    "svdag_alt_table_read": [_P, _P, _U32, _P, _P],
    "svdag_alt_table_sync": [_P, _P],
    "svdag_alt_table_get_stats": [_P, C.POINTER(TableStats), _P],
    "svdag_alt_table_tune": [_P, _P, _U32, _U32, _U32, _P, _P, _P],
    "svdag_alt_table_clear_active": [_P, _P],
    "svdag_alt_table_mark_active": [_P, _P, _U32, _P],
    "svdag_alt_table_free_inactive": [_P, C.POINTER(_U64), _P],
    "svdag_get_stats": [_P, C.POINTER(Stats), _P],
    "svdag_export_level": [_P, _U32, _P, _P, _U64, C.POINTER(_U64), _P],
    "svdag_autotune": [_P, C.POINTER(Edit), _U32, _P, _P, _U32, _U64, _U32, C.POINTER(Tuning), _P],
    "svdag_get_tuning": [_P, C.POINTER(Tuning)],
    "svdag_set_tuning": [_P, C.POINTER(Tuning)],
    "svdag_server_create": [_P, C.POINTER(ServerConfig), C.POINTER(_P)],
    "svdag_server_destroy": [_P],
    "svdag_submit_edit": [_P, C.POINTER(Edit), C.POINTER(_U64)],
    "svdag_submit_frame": [_P, C.POINTER(TraceParams), C.POINTER(_U64)],
    "svdag_poll": [_P, _U64, C.c_int, C.POINTER(RequestResult)],
    "svdag_server_frame": [_P, _P, _U64],
    "svdag_server_counters": [_P, C.POINTER(_U64), C.POINTER(_U64), C.POINTER(_U64)],
    "svdag_server_memory_stats": [_P, C.POINTER(ServerMemory)],
    "svdag_server_replay": [_P, C.POINTER(Edit), _P, _U32, _P, _U32, _P],
    "svdag_submit_undo": [_P, C.c_int, C.POINTER(_U64)],
    "svdag_replay_parse": [C.c_char_p, _U64, C.c_float, _P, _U64, C.POINTER(_U64), C.POINTER(_U64)],
    "svdag_server_replay_actions": [_P, _P, _U64, C.c_double, _P, _P],
    "svdag_save_items": [_P, _P, _U64, _P, _P, C.POINTER(_U64), _P],
    "svdag_shade": [_P, C.POINTER(TraceParams), C.POINTER(ShadeParams), _P, _P, _P, _P, _P],
    "svdag_load_items": [_P, _P, _P, _P, _P],
    "svdag_basic_dag_to_items": [_P, _U64, _U32, _U32, _P, _U64, _P, _P, C.POINTER(_U64)],
    "svdag_v3_to_items": [_P, _U64, _U32, _P, _U64, _P, _P, C.POINTER(_U64)],
    "svdag_items_to_v3": [_P, _P, _P, _U32, _U32, C.c_char_p],
}
EXPORTED = tuple(_PROTOS)

_lib = None


def lib():
    """Loads the in-tree libsvdag.so (never a CPU substitute)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with gpu-svdag-editing_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, args in _PROTOS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.svdag_status_string.restype = C.c_char_p
        L.svdag_abi_version.restype = C.c_uint32
        L.svdag_scene_height.restype = C.c_uint32
        _lib = L
    return _lib


def scene_height(levels: int, x: int, z: int, **terrain) -> int:
    """Surface height of column (x, z) of the procedural terrain (svdag_scene_height)."""
    return lib().svdag_scene_height(C.byref(TerrainParams(**terrain)), levels, x, z)


def _check(status: int, what: str):
    if status != 0:
        raise SvdagError(status, what)


def ptr(x) -> int:
    """Device or host pointer of a torch tensor / numpy array / int."""
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    raise TypeError(type(x))


def stream_ptr(stream) -> int:
    if stream is None:
        return 0
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


# ------------------------------------------------------------------ tools (my_gpu_dag_editors.h)

@dataclass
class MyGpuSphereEditor:
    """MyGpuSphereEditor<isAdding> (my_gpu_dag_editors.h:457-496)."""
    center: tuple
    radius: float
    material: int
    is_adding: bool = True

    def to_edit(self) -> Edit:
        e = Edit(tool=TOOL_SPHERE_ADD if self.is_adding else TOOL_SPHERE_REMOVE, material=self.material)
        e.center[:] = [float(v) for v in self.center]
        e.radius = float(self.radius)
        return e


@dataclass
class MyGpuSphereErosionEditor:
    """MyGpuSphereErosionEditor (my_gpu_dag_editors.h:538-589): inside the sphere, a filled voxel stays
    when more than `threshold` of its 26 neighbours are filled in the DAG before the edit."""
    center: tuple
    radius: float
    threshold: int

    def to_edit(self) -> Edit:
        e = Edit(tool=TOOL_SPHERE_ERODE, material=0, noise_seed=int(self.threshold))
        e.center[:] = [float(v) for v in self.center]
        e.radius = float(self.radius)
        return e


@dataclass
class MyGpuBoxEditor:
    """MyGpuBoxEditor<isAdding> (my_gpu_dag_editors.h:82-119); radius = half extent."""
    center: tuple
    radius: float
    material: int
    is_adding: bool = True

    def to_edit(self) -> Edit:
        e = Edit(tool=TOOL_BOX_ADD if self.is_adding else TOOL_BOX_REMOVE, material=self.material)
        e.center[:] = [float(v) for v in self.center]
        e.radius = float(self.radius)
        return e


@dataclass
class MyGpuSpherePaintEditor:
    """MyGpuSpherePaintEditor (my_gpu_dag_editors.h:498-536); the paint colour only shades."""
    center: tuple
    radius: float
    paint_color: tuple
    material: int

    def to_edit(self) -> Edit:
        e = Edit(tool=TOOL_SPHERE_PAINT, material=self.material)
        e.center[:] = [float(v) for v in self.center]
        e.radius = float(self.radius)
        return e


@dataclass
class MyGpuCopyEditor:
    """MyGpuCopyEditor (my_gpu_dag_editors.h:129-253): pastes the box of half extent `radius` around
    `center` from `source` to `dest` (voxels that are empty in the source keep their old value)."""
    source: tuple
    dest: tuple
    center: tuple
    radius: float
    move: bool = False

    def to_edit(self) -> Edit:
        e = Edit(tool=TOOL_MOVE if self.move else TOOL_COPY, material=0)
        e.src[:] = [float(v) for v in self.source]
        e.dst[:] = [float(v) for v in self.dest]
        e.center[:] = [float(v) for v in self.center]
        e.radius = float(self.radius)
        return e


@dataclass
class MyGpuBoxNoisePaintEditor:
    """Box paint whose material comes from 3D value noise (lattice cell 2^cell_log2 voxels)."""
    center: tuple
    radius: float
    seed: int = 0
    cell_log2: int = 5

    def to_edit(self) -> Edit:
        e = Edit(tool=TOOL_BOX_PAINT_NOISE, material=0, noise_seed=self.seed, noise_cell_log2=self.cell_log2)
        e.center[:] = [float(v) for v in self.center]
        e.radius = float(self.radius)
        return e


# ------------------------------------------------------------------ DAG context

class MyGPUHashDAG:
    """One context: one HBM pool, one slab hash table per level, the root and the undo history."""

    def __init__(self, levels: int, pool_bytes: int = 1 << 30, scratch_bytes: int = 0, device: int = 0,
                 load_factor: int = 0, probe_lanes: int = 0, undo_depth: int = 0, phase_kernels: bool = False,
                 persistent: bool = False):
        cfg = Config(levels=levels, device=device, pool_bytes=pool_bytes, scratch_bytes=scratch_bytes,
                     target_load_factor=load_factor, probe_lanes=probe_lanes, undo_depth=undo_depth,
                     flags=(1 if phase_kernels else 0) | (2 if persistent else 0))
        h = C.c_void_p()
        _check(lib().svdag_create(C.byref(cfg), C.byref(h)), "svdag_create")
        self.h = h
        self.levels = levels

    def free(self):
        if getattr(self, "h", None):
            try:
                lib().svdag_destroy(self.h)
            except Exception:  # interpreter shutdown
                pass
            self.h = None

    __del__ = free

    def leaf_level(self) -> int:
        return self.levels - 2

    def sync(self, stream=None):
        _check(lib().svdag_sync(self.h, stream_ptr(stream)), "svdag_sync")

    def build_terrain(self, seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70,
                      num_structures=0, structure_seed=0, tile_level=0, stream=None):
        p = TerrainParams(seed=seed, octaves=octaves, num_materials=num_materials, min_height_pct=min_height_pct,
                          max_height_pct=max_height_pct, num_structures=num_structures,
                          structure_seed=structure_seed, tile_level=tile_level)
        _check(lib().svdag_build_terrain(self.h, C.byref(p), stream_ptr(stream)), "svdag_build_terrain")

    def edit(self, editor, stream=None):
        e = editor if isinstance(editor, Edit) else editor.to_edit()
        _check(lib().svdag_edit_apply(self.h, C.byref(e), stream_ptr(stream)), "svdag_edit_apply")

    def edit_batch(self, editors, stream=None) -> int:
        """Batched form: all edits in one persistent launch. Returns the number of records
        (a move yields two)."""
        arr = (Edit * len(editors))(*[e if isinstance(e, Edit) else e.to_edit() for e in editors])
        _check(lib().svdag_edit_apply_many(self.h, arr, len(editors), stream_ptr(stream)), "svdag_edit_apply_many")
        return sum(2 if e.tool == TOOL_MOVE else 1 for e in arr)

    def edit_records(self, count: int, stream=None):
        out = (EditRecord * count)()
        _check(lib().svdag_edit_records(self.h, out, count, stream_ptr(stream)), "svdag_edit_records")
        return list(out)

    def last_edit_phase_times(self, stream=None):
        """GPU timestamps (ns) at the phase barriers of the last persistent-kernel edit."""
        buf = np.zeros(64, dtype=np.uint64)
        n = C.c_uint32()
        _check(lib().svdag_last_edit_phase_times(self.h, buf.ctypes.data, 64, C.byref(n), stream_ptr(stream)),
               "svdag_last_edit_phase_times")
        return buf[: n.value].copy()

    def last_edit_stats(self, stream=None) -> EditStats:
        st = EditStats()
        _check(lib().svdag_last_edit_stats(self.h, C.byref(st), stream_ptr(stream)), "svdag_last_edit_stats")
        return st

    def get_first_node_index(self, stream=None) -> int:
        r = C.c_uint32()
        _check(lib().svdag_get_root(self.h, C.byref(r), stream_ptr(stream)), "svdag_get_root")
        return r.value

    def undo(self, stream=None):
        _check(lib().svdag_undo(self.h, stream_ptr(stream)), "svdag_undo")

    def redo(self, stream=None):
        _check(lib().svdag_redo(self.h, stream_ptr(stream)), "svdag_redo")

    def garbage_collect(self, stream=None, keep_history: bool = False):
        """MyGPUHashDAGUndoRedo::garbageCollect: frees what the root cannot reach and clears the
        history; keep_history=True marks from every undo/redo root too and keeps the history."""
        if keep_history:
            _check(lib().svdag_gc_keep_history(self.h, stream_ptr(stream)), "svdag_gc_keep_history")
        else:
            _check(lib().svdag_gc(self.h, stream_ptr(stream)), "svdag_gc")

    def stats(self, stream=None) -> Stats:
        s = Stats()
        _check(lib().svdag_get_stats(self.h, C.byref(s), stream_ptr(stream)), "svdag_get_stats")
        return s

    def table(self, level: int) -> "HashTable":
        t = C.c_void_p()
        _check(lib().svdag_level_table(self.h, level, C.byref(t)), "svdag_level_table")
        return HashTable(self, t, KIND_LEAF if level == self.leaf_level() else KIND_NODE, owned=False)

    def create_table(self, kind: int, buckets_per_size) -> "HashTable":
        b = np.ascontiguousarray(buckets_per_size, dtype=np.uint32)
        assert b.size == NUM_SIZE_CLASSES
        t = C.c_void_p()
        _check(lib().svdag_table_create(self.h, kind, b.ctypes.data, C.byref(t)), "svdag_table_create")
        return HashTable(self, t, kind, owned=True)

    def trace(self, params: TraceParams, out, stream=None):
        """Writes width*height hit records into the device buffer `out` (68 bytes each)."""
        _check(lib().svdag_trace_primary(self.h, C.byref(params), ptr(out), stream_ptr(stream)), "svdag_trace_primary")

    def sample_voxels(self, xyz_dev, count: int, out_dev, stream=None):
        _check(lib().svdag_sample_voxels(self.h, ptr(xyz_dev), count, ptr(out_dev), stream_ptr(stream)),
               "svdag_sample_voxels")

    def autotune(self, edits=(), keys=None, offsets=None, n_keys=0, total_words=0, kind=0, stream=None) -> "Tuning":
        """Autotuner (svdag_autotune): key sample -> load factor and lanes per key; edit sample (applied
        for real) -> which small edits use the persistent kernel."""
        arr = (Edit * max(len(edits), 1))(*[e if isinstance(e, Edit) else e.to_edit() for e in edits])
        t = Tuning()
        _check(lib().svdag_autotune(self.h, arr, len(edits), ptr(keys), ptr(offsets), n_keys, total_words, kind,
                                    C.byref(t), stream_ptr(stream)), "svdag_autotune")
        return t

    def tuning(self) -> "Tuning":
        t = Tuning()
        _check(lib().svdag_get_tuning(self.h, C.byref(t)), "svdag_get_tuning")
        return t

    def set_tuning(self, t: "Tuning"):
        _check(lib().svdag_set_tuning(self.h, C.byref(t)), "svdag_set_tuning")

    def export_level(self, level: int):
        """(handles uint32[n], words uint32[n, 10]) of every item in the level table."""
        n = C.c_uint64()
        _check(lib().svdag_export_level(self.h, level, None, None, 0, C.byref(n), None), "svdag_export_level")
        cap = n.value
        handles = np.zeros(cap, dtype=np.uint32)
        words = np.zeros((cap, MAX_ITEM_WORDS), dtype=np.uint32)
        if cap:
            _check(lib().svdag_export_level(self.h, level, handles.ctypes.data, words.ctypes.data, cap, C.byref(n),
                                            None), "svdag_export_level")
        return handles[: n.value], words[: n.value]

    def save_items(self, stream=None) -> "ItemSnapshot":
        """The items reachable from the root as an item snapshot (svdag_save_items), the portable form
        that writeTo converts to the reference's file."""
        nl = self.levels - 1
        lw, li, total = np.zeros(nl, np.uint64), np.zeros(nl, np.uint64), C.c_uint64()
        words = np.zeros(0, np.uint32)
        while True:
            st = lib().svdag_save_items(self.h, words.ctypes.data if len(words) else None, len(words), lw.ctypes.data,
                                        li.ctypes.data, C.byref(total), stream_ptr(stream))
            if st == 2 and total.value > len(words):
                words = np.zeros(total.value, np.uint32)
                continue
            _check(st, "svdag_save_items")
            return ItemSnapshot(self.levels, words[: total.value], lw, li)

    def load_items(self, snap: "ItemSnapshot", stream=None):
        """Replaces the DAG by an item snapshot (svdag_load_items), the portable form that readFrom
        converts the reference's file to."""
        if snap.levels != self.levels:
            raise SvdagError(1, f"svdag_load_items: snapshot of {snap.levels} levels, DAG of {self.levels}")
        w = np.ascontiguousarray(snap.words, dtype=np.uint32)
        lw = np.ascontiguousarray(snap.level_words, dtype=np.uint64)
        li = np.ascontiguousarray(snap.level_items, dtype=np.uint64)
        _check(lib().svdag_load_items(self.h, w.ctypes.data if len(w) else None, lw.ctypes.data, li.ctypes.data,
                                      stream_ptr(stream)), "svdag_load_items")

    def write_to(self, path: str):
        """Writes the DAG as a portable item snapshot file (ItemSnapshot.write)."""
        self.save_items().write(path)

    def read_from(self, path: str):
        """Replaces the DAG by an item snapshot file (ItemSnapshot.read)."""
        self.load_items(ItemSnapshot.read(path))

    def writeTo(self, path: str, memory_type: int = V3_GPU_MALLOC):
        """MyGPUHashDAG::writeTo (my_gpu_hash_dag.cu:158-165): the DAG as the reference's own version-3
        file, which the reference's readFrom loads (svdag_save_items, then svdag_items_to_v3)."""
        items_to_v3(self.save_items(), path, memory_type)

    def readFrom(self, path: str):
        """MyGPUHashDAG::readFrom (my_gpu_hash_dag.cu:167-177): replaces the DAG by a version-3 file
        the reference wrote (svdag_v3_to_items, then svdag_load_items)."""
        self.load_items(v3_to_items(path, self.levels))

    def load_basic_dag(self, path: str, material: int = 0) -> "BasicDAGFile":
        """Loads a BasicDAG geometry file of the reference (BasicDAGFactory::load_dag_from_file,
        basic_dag.cpp:108-122) with every voxel of `material`; returns the file's header."""
        f = BasicDAGFile.read(path)
        if f.levels != self.levels:
            raise SvdagError(1, f"BasicDAG of {f.levels} levels, DAG of {self.levels}")
        self.load_items(basic_dag_to_items(f.data, f.levels, material))
        return f


@dataclass
class ItemSnapshot:
    """Per-level item lists of a DAG (include/svdag.h, "import and export"). The file form is
    b"SVDAGIT1", u32 version 1, u32 levels, u64 level_words[levels-1], u64 level_items[levels-1],
    then the words, all little-endian."""
    levels: int
    words: np.ndarray
    level_words: np.ndarray
    level_items: np.ndarray

    MAGIC = b"SVDAGIT1"

    def write(self, path: str):
        with open(path, "wb") as f:
            f.write(self.MAGIC)
            f.write(np.array([1, self.levels], dtype="<u4").tobytes())
            f.write(np.asarray(self.level_words, dtype="<u8").tobytes())
            f.write(np.asarray(self.level_items, dtype="<u8").tobytes())
            f.write(np.asarray(self.words, dtype="<u4").tobytes())

    @classmethod
    def read(cls, path: str) -> "ItemSnapshot":
        with open(path, "rb") as f:
            data = f.read()
        if data[:8] != cls.MAGIC:
            raise SvdagError(1, f"{path}: not an item snapshot")
        version, levels = np.frombuffer(data, "<u4", 2, 8)
        if version != 1 or not 4 <= levels <= MAX_LEVELS:
            raise SvdagError(1, f"{path}: version {version}, levels {levels}")
        nl = int(levels) - 1
        lw = np.frombuffer(data, "<u8", nl, 16).copy()
        li = np.frombuffer(data, "<u8", nl, 16 + 8 * nl).copy()
        at = 16 + 16 * nl
        total = int(lw.sum())
        if len(data) != at + 4 * total:
            raise SvdagError(1, f"{path}: {len(data)} bytes, expected {at + 4 * total}")
        return cls(int(levels), np.frombuffer(data, "<u4", total, at).copy(), lw, li)


@dataclass
class BasicDAGFile:
    """The reference's BasicDAG file (BasicDAGFactory::save_dag_to_file, basic_dag.cpp:95-106, through
    FileWriter, serializer.h:12-61): DAGInfo as six doubles (AABB min, max), u32 levels, u64 word
    count, then the node words."""
    bounds_min: tuple
    bounds_max: tuple
    levels: int
    data: np.ndarray

    def write(self, path: str):
        with open(path, "wb") as f:
            f.write(np.array(list(self.bounds_min) + list(self.bounds_max), dtype="<f8").tobytes())
            f.write(np.array([self.levels], dtype="<u4").tobytes())
            f.write(np.array([len(self.data)], dtype="<u8").tobytes())
            f.write(np.asarray(self.data, dtype="<u4").tobytes())

    @classmethod
    def read(cls, path: str) -> "BasicDAGFile":
        with open(path, "rb") as f:
            data = f.read()
        if len(data) < 60:
            raise SvdagError(1, f"{path}: too short for a BasicDAG file")
        b = np.frombuffer(data, "<f8", 6, 0)
        levels = int(np.frombuffer(data, "<u4", 1, 48)[0])
        n = int(np.frombuffer(data, "<u8", 1, 52)[0])
        if len(data) != 60 + 4 * n:
            raise SvdagError(1, f"{path}: {len(data)} bytes, expected {60 + 4 * n}")
        return cls(tuple(float(v) for v in b[:3]), tuple(float(v) for v in b[3:]), levels,
                   np.frombuffer(data, "<u4", n, 60).copy())


def basic_dag_to_items(data, levels: int, material: int = 0) -> ItemSnapshot:
    """BasicDAG node words -> item snapshot, every voxel of `material` (svdag_basic_dag_to_items, a
    host function: create_dag_cpu without colour import, my_gpu_hash_dag_factory.cpp:316-418)."""
    d = np.ascontiguousarray(data, dtype=np.uint32)
    nl = levels - 1
    lw, li, total = np.zeros(nl, np.uint64), np.zeros(nl, np.uint64), C.c_uint64()
    st = lib().svdag_basic_dag_to_items(d.ctypes.data, len(d), levels, material, None, 0, lw.ctypes.data, li.ctypes.data,
                                        C.byref(total))
    if st not in (0, 2):
        _check(st, "svdag_basic_dag_to_items")
    words = np.zeros(max(total.value, 1), np.uint32)
    _check(lib().svdag_basic_dag_to_items(d.ctypes.data, len(d), levels, material, words.ctypes.data, len(words),
                                          lw.ctypes.data, li.ctypes.data, C.byref(total)), "svdag_basic_dag_to_items")
    return ItemSnapshot(levels, words[: total.value], lw, li)


def v3_to_items(path: str, levels: int) -> ItemSnapshot:
    """A version-3 DAG file of the reference (MyGPUHashDAG::writeTo) -> item snapshot
    (svdag_v3_to_items, a host function). The file is mapped, not read into memory."""
    size = os.path.getsize(path)
    data = np.memmap(path, dtype=np.uint8, mode="r") if size else np.zeros(0, np.uint8)
    base = data.ctypes.data if size else None
    nl = levels - 1
    lw, li, total = np.zeros(nl, np.uint64), np.zeros(nl, np.uint64), C.c_uint64()
    st = lib().svdag_v3_to_items(base, size, levels, None, 0, lw.ctypes.data, li.ctypes.data, C.byref(total))
    if st not in (0, 2):
        _check(st, "svdag_v3_to_items")
    words = np.zeros(max(total.value, 1), np.uint32)
    _check(lib().svdag_v3_to_items(base, size, levels, words.ctypes.data, len(words), lw.ctypes.data, li.ctypes.data,
                                   C.byref(total)), "svdag_v3_to_items")
    del data
    return ItemSnapshot(levels, words[: total.value], lw, li)


def items_to_v3(snap: ItemSnapshot, path: str, memory_type: int = V3_GPU_MALLOC):
    """Item snapshot -> the reference's version-3 DAG file (svdag_items_to_v3, a host function);
    `memory_type` is the EMemoryType the file records (V3_*)."""
    words = np.ascontiguousarray(snap.words, dtype=np.uint32)
    lw = np.ascontiguousarray(snap.level_words, dtype=np.uint64)
    li = np.ascontiguousarray(snap.level_items, dtype=np.uint64)
    _check(lib().svdag_items_to_v3(words.ctypes.data if len(words) else None, lw.ctypes.data, li.ctypes.data, snap.levels,
                                   memory_type, os.fsencode(path)), "svdag_items_to_v3")


class HashTable:
    """Batched find/add over one slab hash table (MyGPUHashDAG::find_/add_{node,leaf}_as_warp)."""

    def __init__(self, dag: MyGPUHashDAG, handle, kind: int, owned: bool):
        self.dag, self.h, self.kind, self.owned = dag, handle, kind, owned

    def _op(self, fn, keys, offsets, count, total_words, out, lanes, stream):
        _check(fn(self.h, ptr(keys), ptr(offsets), count, total_words, ptr(out), lanes, stream_ptr(stream)), fn.__name__)

    def add(self, keys, offsets, count, total_words, out, lanes=0, stream=None):
        self._op(lib().svdag_table_add, keys, offsets, count, total_words, out, lanes, stream)

    def find(self, keys, offsets, count, total_words, out, lanes=0, stream=None):
        self._op(lib().svdag_table_find, keys, offsets, count, total_words, out, lanes, stream)

    def find_or_add(self, keys, offsets, count, total_words, out, lanes=0, stream=None):
        self._op(lib().svdag_table_find_or_add, keys, offsets, count, total_words, out, lanes, stream)

    def find_or_add_static(self, keys, offsets, count, total_words, out, lanes=0, stream=None):
        """find_or_add without any allocation: scratch is a fixed array inside the library
        (at most 65536 keys per call; calls that overlap on the GPU must be serialised)."""
        self._op(lib().svdag_table_find_or_add_static, keys, offsets, count, total_words, out, lanes, stream)

    def read(self, handles, count, out_words, stream=None):
        _check(lib().svdag_table_read(self.h, ptr(handles), count, ptr(out_words), stream_ptr(stream)),
               "svdag_table_read")

    def stats(self, stream=None) -> TableStats:
        s = TableStats()
        _check(lib().svdag_table_get_stats(self.h, C.byref(s), stream_ptr(stream)), "svdag_table_get_stats")
        return s

    def destroy(self):
        if self.owned and self.h:
            lib().svdag_table_destroy(self.h)
            self.h = None


TABLE_LAYOUT_TICKET_BOARD, TABLE_LAYOUT_ATOMIC64, TABLE_LAYOUT_ACCELERATION, TABLE_LAYOUT_INDIVIDUAL_CHAINING = 1, 2, 3, 4


class AltHashTable:
    """A table of fixed-size items in one of the reference's alternative layouts (TicketBoardHashTable,
    Atomic64HashTable, AccelerationHashTable, IndividualChainingHashTable), on the GPU of `dag`, in an
    allocation of its own. Keys are `item_words` words back to back; add stores every key in a
    fresh slot, duplicates included; adds and finds must not overlap in time."""

    def __init__(self, dag: MyGPUHashDAG, layout: int, item_words: int, num_buckets: int, reserved_items: int):
        self.dag, self.layout, self.item_words = dag, layout, item_words
        t = C.c_void_p()
        _check(lib().svdag_alt_table_create(dag.h, layout, item_words, num_buckets, reserved_items, C.byref(t)),
               "svdag_alt_table_create")
        self.h = t

    @classmethod
    def allocate(cls, dag: MyGPUHashDAG, layout: int, numBuckets: int, numReservedElements: int, itemSizeInU32: int):
        """Table::allocate(numBuckets, numReservedElements, itemSizeInU32)."""
        return cls(dag, layout, itemSizeInU32, numBuckets, numReservedElements)

    def add(self, keys, count, out, lanes=0, stream=None):
        _check(lib().svdag_alt_table_add(self.h, ptr(keys), count, ptr(out), lanes, stream_ptr(stream)), "svdag_alt_table_add")

    def find(self, keys, count, out, lanes=0, stream=None):
        _check(lib().svdag_alt_table_find(self.h, ptr(keys), count, ptr(out), lanes, stream_ptr(stream)),
               "svdag_alt_table_find")

    def read(self, handles, count, out_words, stream=None):
        _check(lib().svdag_alt_table_read(self.h, ptr(handles), count, ptr(out_words), stream_ptr(stream)),
               "svdag_alt_table_read")

    def sync(self, stream=None):
        """Waits for the stream; raises the first device-side error latched since the last sync."""
        _check(lib().svdag_alt_table_sync(self.h, stream_ptr(stream)), "svdag_alt_table_sync")

    def stats(self, stream=None) -> TableStats:
        s = TableStats()
        _check(lib().svdag_alt_table_get_stats(self.h, C.byref(s), stream_ptr(stream)), "svdag_alt_table_get_stats")
        return s

    def clearActiveFlags(self, stream=None):
        _check(lib().svdag_alt_table_clear_active(self.h, stream_ptr(stream)), "svdag_alt_table_clear_active")

    def markAsActive(self, handles, count, stream=None):
        _check(lib().svdag_alt_table_mark_active(self.h, ptr(handles), count, stream_ptr(stream)),
               "svdag_alt_table_mark_active")

    def freeInactiveItems(self, stream=None) -> int:
        """Frees every stored item not marked since clearActiveFlags; returns how many."""
        n = C.c_uint64()
        _check(lib().svdag_alt_table_free_inactive(self.h, C.byref(n), stream_ptr(stream)), "svdag_alt_table_free_inactive")
        return n.value

    def destroy(self):
        if self.h:
            lib().svdag_alt_table_destroy(self.h)
            self.h = None


class AltTuning(C.Structure):
    _fields_ = [("layout", _U32), ("lanes", _U32), ("add_ms", C.c_float), ("find_ms", C.c_float)]


ALT_TUNING_CANDIDATES = 7


def alt_table_tune(dag: MyGPUHashDAG, keys, count: int, item_words: int, items_per_bucket: int = 0, stream=None):
    """svdag_alt_table_tune: (best candidate, all candidates) among the alternative layouts and launch
    forms, measured on `count` keys of `item_words` words (a device array)."""
    best = AltTuning()
    every = (AltTuning * ALT_TUNING_CANDIDATES)()
    _check(lib().svdag_alt_table_tune(dag.h, ptr(keys), count, item_words, items_per_bucket, C.addressof(best),
                                      C.addressof(every), stream_ptr(stream)), "svdag_alt_table_tune")
    return best, list(every)


def TicketBoardHashTable(dag, numBuckets, numReservedElements, itemSizeInU32):
    return AltHashTable.allocate(dag, TABLE_LAYOUT_TICKET_BOARD, numBuckets, numReservedElements, itemSizeInU32)


def Atomic64HashTable(dag, numBuckets, numReservedElements, itemSizeInU32):
    return AltHashTable.allocate(dag, TABLE_LAYOUT_ATOMIC64, numBuckets, numReservedElements, itemSizeInU32)


def AccelerationHashTable(dag, numBuckets, numReservedElements, itemSizeInU32):
    return AltHashTable.allocate(dag, TABLE_LAYOUT_ACCELERATION, numBuckets, numReservedElements, itemSizeInU32)


def IndividualChainingHashTable(dag, numBuckets, numReservedElements, itemSizeInU32):
    return AltHashTable.allocate(dag, TABLE_LAYOUT_INDIVIDUAL_CHAINING, numBuckets, numReservedElements, itemSizeInU32)


class MyGPUHashDAGUndoRedo:
    """MyGPUHashDAGUndoRedo (my_gpu_base_dag.h:16-82); the history itself lives on the device."""

    def undo(self, dag: MyGPUHashDAG, stream=None):
        dag.undo(stream)

    def redo(self, dag: MyGPUHashDAG, stream=None):
        dag.redo(stream)

    def garbageCollect(self, dag: MyGPUHashDAG, stream=None):
        dag.garbage_collect(stream)


def editMyHashDag(editor, dag: MyGPUHashDAG, undoRedo: MyGPUHashDAGUndoRedo | None = None, stream=None):
    """editMyHashDag<Editor> (my_gpu_hash_dag_edits.h:12-13): applies one tool; the undo frame is
    recorded on the device, so `undoRedo` is accepted only for signature compatibility."""
    dag.edit(editor, stream)


# ------------------------------------------------------------------ camera (dag_tracer.cu:59-101)

def get_trace_params(position, target, width: int, height: int, fov_degrees: float = 60.0,
                     levels: int | None = None, bounds_min=(0.0, 0.0, 0.0), bounds_max=None) -> TraceParams:
    """Ray basis of a look-at camera in double precision. With bounds given, world coordinates are
    scaled to the [0, 2^levels) voxel grid as get_trace_params does; by default they already are voxels."""
    pos = np.asarray(position, dtype=np.float64)
    f = np.asarray(target, dtype=np.float64) - pos
    f = f / math.sqrt(float(np.dot(f, f)))
    wu = np.array([0.0, 0.0, 1.0]) if abs(f[1]) > 0.999 else np.array([0.0, 1.0, 0.0])
    r = np.cross(f, wu)
    r = r / math.sqrt(float(np.dot(r, r)))
    u = np.cross(r, f)
    fov = fov_degrees / 2.0 * (math.pi / 180.0)
    aspect = float(width) / float(height)
    X = r * math.sin(fov) * aspect
    Y = u * math.sin(fov)
    Z = f * math.cos(fov)
    bl, br, tl = pos + Z - Y - X, pos + Z - Y + X, pos + Z + Y - X
    if bounds_max is not None:
        bmin, bmax = np.asarray(bounds_min, dtype=np.float64), np.asarray(bounds_max, dtype=np.float64)
        scale = float(1 << levels) / (bmax - bmin)
        pos, bl, br, tl = [(v - bmin) * scale for v in (pos, bl, br, tl)]
    p = TraceParams()
    p.camera[:] = list(pos)
    p.ray_min[:] = list(bl)
    p.ray_ddx[:] = list((br - bl) * (1.0 / width))
    p.ray_ddy[:] = list((tl - bl) * (1.0 / height))
    p.width, p.height = width, height
    return p


class DAGTracer:
    """DAGTracer (dag_tracer.h): owns the per-pixel hit buffer (a device tensor of 68-byte records)."""

    def __init__(self, width: int, height: int, device: str = "cuda"):
        import torch
        self.width, self.height = width, height
        self.hits = torch.empty(width * height * HIT_DTYPE.itemsize, dtype=torch.uint8, device=device)

    def resolve_paths(self, params: TraceParams, dag: MyGPUHashDAG, stream=None):
        assert params.width == self.width and params.height == self.height
        dag.trace(params, self.hits, stream)

    def hits_numpy(self) -> np.ndarray:
        return self.hits.cpu().numpy().view(HIT_DTYPE)

    def resolve_lighting(self, params: TraceParams, dag: MyGPUHashDAG, shade: ShadeParams, want_surfaces: bool = False,
                         stream=None):
        """Colours, shadows, ambient occlusion and lighting of the last resolve_paths
        (DAGTracer::resolve_colors / resolve_shadows / resolve_ambient_occlusion / resolve_lighting,
        dag_tracer.cu:136-250) in one launch: returns the sRGB8 image as a device tensor, plus the sun
        and AO surfaces with want_surfaces."""
        import torch
        n = self.width * self.height
        self.colors = torch.empty(n, dtype=torch.int32, device=self.hits.device)
        sun = torch.empty(n, dtype=torch.float32, device=self.hits.device) if want_surfaces else None
        ao = torch.empty(n, dtype=torch.float32, device=self.hits.device) if want_surfaces else None
        _check(lib().svdag_shade(dag.h, C.byref(params), C.byref(shade), ptr(self.hits), ptr(self.colors),
                                 ptr(sun) if sun is not None else None, ptr(ao) if ao is not None else None,
                                 stream_ptr(stream)), "svdag_shade")
        return (self.colors, sun, ao) if want_surfaces else self.colors


class Server:
    """The serving form: a native request loop over a resident DAG (svdag_server_*). With
    plain=True it is the per-edit baseline: one request at a time, each edit followed by a frame."""

    def __init__(self, dag: MyGPUHashDAG, frame: TraceParams, max_batch: int = 256, max_inflight: int = 2,
                 memory_cap_bytes: int = 0, plain: bool = False, copy_frames: bool = False, full_frames: bool = False,
                 gc_threshold_bytes: int = 0, gc: bool = True):
        self.dag = dag
        self.frame_params = frame
        flags = ((SERVE_PLAIN if plain else 0) | (SERVE_COPY_FRAMES if copy_frames else 0)
                 | (SERVE_FULL_FRAMES if full_frames else 0) | (0 if gc else SERVE_NO_GC))
        cfg = ServerConfig(max_batch=max_batch, max_inflight=max_inflight, memory_cap_bytes=memory_cap_bytes,
                           frame=frame, flags=flags, gc_threshold_bytes=gc_threshold_bytes)
        h = C.c_void_p()
        _check(lib().svdag_server_create(dag.h, C.byref(cfg), C.byref(h)), "svdag_server_create")
        self.h = h

    def submit_edit(self, editor) -> int:
        e = editor if isinstance(editor, Edit) else editor.to_edit()
        t = C.c_uint64()
        _check(lib().svdag_submit_edit(self.h, C.byref(e), C.byref(t)), "svdag_submit_edit")
        return t.value

    def submit_frame(self, params: TraceParams | None = None) -> int:
        t = C.c_uint64()
        _check(lib().svdag_submit_frame(self.h, C.byref(params) if params is not None else None, C.byref(t)),
               "svdag_submit_frame")
        return t.value

    def poll(self, ticket: int, wait: bool = True):
        """RequestResult, or None while not visible (wait=False)."""
        r = RequestResult()
        st = lib().svdag_poll(self.h, ticket, 1 if wait else 0, C.byref(r))
        if st == 8 and not wait:
            return None
        _check(st, "svdag_poll")
        return r

    def frame(self) -> np.ndarray:
        n = self.frame_params.width * self.frame_params.height
        out = np.zeros(n, dtype=HIT_DTYPE)
        _check(lib().svdag_server_frame(self.h, out.ctypes.data, n), "svdag_server_frame")
        return out

    def replay(self, edits, edit_times, frame_times=()) -> np.ndarray:
        """Submits edit i at edit_times[i] s and frame j at frame_times[j] s after the call starts;
        returns the results (edits first, then frames) once all are visible."""
        arr = (Edit * max(len(edits), 1))(*[e if isinstance(e, Edit) else e.to_edit() for e in edits])
        et = np.ascontiguousarray(edit_times, dtype=np.float64)
        ft = np.ascontiguousarray(frame_times, dtype=np.float64)
        out = np.zeros(len(edits) + len(ft), dtype=RESULT_DTYPE)
        _check(lib().svdag_server_replay(self.h, arr, et.ctypes.data, len(edits), ft.ctypes.data, len(ft),
                                         out.ctypes.data), "svdag_server_replay")
        return out

    def counters(self) -> dict:
        """Frames traced whole and incrementally so far, bytes of frames copied to the host."""
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _check(lib().svdag_server_counters(self.h, C.byref(a), C.byref(b), C.byref(c)), "svdag_server_counters")
        return {"frames_whole": a.value, "frames_incremental": b.value, "frame_bytes_to_host": c.value}

    def memory(self) -> dict:
        """Bytes in use, cap and threshold, in-loop collections, edits rejected and failed."""
        m = ServerMemory()
        _check(lib().svdag_server_memory_stats(self.h, C.byref(m)), "svdag_server_memory_stats")
        return {f: getattr(m, f) for f, _ in ServerMemory._fields_}

    def submit_undo(self, redo: bool = False) -> int:
        t = C.c_uint64()
        _check(lib().svdag_submit_undo(self.h, 1 if redo else 0, C.byref(t)), "svdag_submit_undo")
        return t.value

    def replay_actions(self, actions, frame_period_s: float = 0.0, frames=None) -> np.ndarray:
        """Serves parsed replay actions (parse_replay), one recorded frame every frame_period_s
        seconds; `frames` (one TraceParams per EndFrame, e.g. replay_frames) overrides the configured
        camera. Returns one result per action (ticket 0 for actions that are not requests)."""
        n = len(actions)
        out = np.zeros(n, dtype=RESULT_DTYPE)
        fr = None
        if frames is not None:
            fr = (TraceParams * max(len(frames), 1))(*frames)
            if len(frames) < sum(1 for a in actions if a.kind == REPLAY_END_FRAME):
                raise SvdagError(1, "replay_actions: one frame per EndFrame")
        _check(lib().svdag_server_replay_actions(self.h, C.addressof(actions) if n else None, n, float(frame_period_s), fr,
                                                 out.ctypes.data), "svdag_server_replay_actions")
        return out

    def close(self):
        if getattr(self, "h", None):
            h, self.h = self.h, None
            _check(lib().svdag_server_destroy(h), "svdag_server_destroy")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---------------------------------------------------------------- recorded edit sessions

def replay_scale(scene_depth: int, replay_depth: int) -> float:
    """scalingFactor of replay.cpp:10: replay positions are voxels of a 2^replay_depth grid."""
    return float(np.float32(float(1 << scene_depth)) / np.float32(float(1 << replay_depth)))


def parse_replay(text, scale: float = 1.0):
    """Parses a reference replay file's text (ReplayManager::load_csv, replay.h:650-683) into a
    ctypes array of ReplayAction, edits scaled by `scale` (svdag_replay_parse)."""
    data = text.encode() if isinstance(text, str) else bytes(text)
    count, bad = C.c_uint64(), C.c_uint64()
    st = lib().svdag_replay_parse(data, len(data), scale, None, 0, C.byref(count), C.byref(bad))
    if st != 0:
        raise SvdagError(st, f"svdag_replay_parse (line {bad.value})")
    arr = (ReplayAction * max(count.value, 1))()
    _check(lib().svdag_replay_parse(data, len(data), scale, C.addressof(arr), count.value, C.byref(count), None),
           "svdag_replay_parse")
    return (ReplayAction * count.value).from_buffer(arr) if count.value else (ReplayAction * 0)()


def view_trace_params(position, rotation, width: int, height: int, levels: int, bounds_min, bounds_max,
                      fov_degrees: float = 60.0) -> TraceParams:
    """Trace parameters of the reference's CameraView (camera_view.h: right = -row 0, up = row 1,
    forward = row 2 of the rotation) through get_trace_params (dag_tracer.cu:59-101), world
    coordinates mapped from [bounds_min, bounds_max] onto the 2^levels voxel grid."""
    pos = np.asarray(position, dtype=np.float32).astype(np.float64)
    m = np.asarray(rotation, dtype=np.float32).reshape(3, 3).astype(np.float64)
    right, up, fwd = -m[0], m[1], m[2]
    fov = fov_degrees / 2.0 * (math.pi / 180.0)
    aspect = float(width) / float(height)
    X = right * math.sin(fov) * aspect
    Y = up * math.sin(fov)
    Z = fwd * math.cos(fov)
    bl, br, tl = pos + Z - Y - X, pos + Z - Y + X, pos + Z + Y - X
    bmin, bmax = np.asarray(bounds_min, dtype=np.float64), np.asarray(bounds_max, dtype=np.float64)
    scale = float(1 << levels) / (bmax - bmin)
    pos, bl, br, tl = [(v - bmin) * scale for v in (pos, bl, br, tl)]
    p = TraceParams()
    p.camera[:] = list(pos)
    p.ray_min[:] = list(bl)
    p.ray_ddx[:] = list((br - bl) * (1.0 / width))
    p.ray_ddy[:] = list((tl - bl) * (1.0 / height))
    p.width, p.height = width, height
    return p


def replay_frames(actions, width: int, height: int, levels: int, bounds_min, bounds_max, position=(0.0, 0.0, 0.0),
                  rotation=(1, 0, 0, 0, 1, 0, 0, 0, 1)) -> list:
    """One TraceParams per EndFrame, from the camera the SetLocation/SetRotation actions before it
    left (the reference's view starts at the origin with the identity rotation, camera_view.h)."""
    pos, rot = list(position), list(rotation)
    out = []
    for a in actions:
        if a.kind == REPLAY_CAMERA_LOCATION:
            pos = list(a.camera[:3])
        elif a.kind == REPLAY_CAMERA_ROTATION:
            rot = list(a.camera[:9])
        elif a.kind == REPLAY_END_FRAME:
            out.append(view_trace_params(pos, rot, width, height, levels, bounds_min, bounds_max))
    return out
