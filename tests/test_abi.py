"""The C ABI library builds, loads and exports every entry point include/svdag.h declares."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "svdag.h")).read()
    return sorted(set(re.findall(r"^\s*(?:svdag_status|const char\*|uint32_t)\s+(svdag_\w+)\s*\(", text, re.M)))


def test_every_declared_symbol_is_exported(svdag_lib):
    names = declared_symbols()
    assert len(names) >= 25
    out = subprocess.check_output(["nm", "-D", "--defined-only", svdag_lib.LIB_PATH], text=True)
    exported = set(re.findall(r" T (svdag_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    assert set(names) == set(svdag_lib.EXPORTED)


def test_library_loads_and_reports_version(svdag_lib):
    L = svdag_lib.lib()
    assert L.svdag_abi_version() == 2
    assert L.svdag_status_string(2).decode().startswith("out of memory")


def test_struct_layouts(svdag_lib):
    s = svdag_lib
    assert s.HIT_DTYPE.itemsize == 68  # Tracer::SurfaceInteraction
    assert C.sizeof(s.Edit) == 56
    assert C.sizeof(s.Config) == 40
    assert C.sizeof(s.TraceParams) == 104
    assert C.sizeof(s.TerrainParams) == 32
    assert C.sizeof(s.ServerConfig) == 136
    assert C.sizeof(s.ServerMemory) == 72
    assert C.sizeof(s.RequestResult) == 48
    assert C.sizeof(s.Tuning) == 40
    assert C.sizeof(s.AltTuning) == 16  # svdag_alt_tuning


def test_invalid_arguments_are_rejected(svdag_lib):
    L = svdag_lib.lib()
    cfg = svdag_lib.Config(levels=3)  # below SVDAG_MIN_LEVELS
    h = C.c_void_p()
    assert L.svdag_create(C.byref(cfg), C.byref(h)) == 1
    cfg = svdag_lib.Config(levels=10, probe_lanes=3)
    assert L.svdag_create(C.byref(cfg), C.byref(h)) == 1
    assert L.svdag_destroy(None) == 1
    assert L.svdag_edit_apply(None, None, None) == 1
    # alternative-layout tables: null handles are rejected before any CUDA call
    t = C.c_void_p()
    assert L.svdag_alt_table_create(None, 1, 2, 16, 0, C.byref(t)) == 1
    for f in (L.svdag_alt_table_add, L.svdag_alt_table_find):
        assert f(None, None, 0, None, 1, None) == 1
    assert L.svdag_alt_table_read(None, None, 0, None, None) == 1
    assert L.svdag_alt_table_sync(None, None) == 1
    assert L.svdag_alt_table_get_stats(None, None, None) == 1
    assert L.svdag_alt_table_destroy(None) == 1
    assert L.svdag_alt_table_tune(None, None, 0, 2, 0, None, None, None) == 1
    assert L.svdag_alt_table_clear_active(None, None) == 1
    assert L.svdag_alt_table_mark_active(None, None, 0, None) == 1
    assert L.svdag_alt_table_free_inactive(None, None, None) == 1


def test_no_cpu_fallback_without_device(svdag_lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(svdag_lib.SvdagError) as e:
        svdag_lib.MyGPUHashDAG(10)
    assert e.value.status == 6  # SVDAG_ERR_NO_DEVICE


def test_header_is_c11_and_the_binding_lays_out_structs_alike(svdag_lib, tmp_path):
    """include/svdag.h compiles as strict C11, every ctypes structure of the Python binding has the
    size and field offsets a C compiler gives the header's struct, and a C program that takes the
    address of every exported function links against libsvdag.so."""
    import shutil

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    s = svdag_lib
    pairs = {"svdag_config": s.Config, "svdag_terrain_params": s.TerrainParams, "svdag_edit": s.Edit,
             "svdag_edit_stats": s.EditStats, "svdag_edit_record": s.EditRecord, "svdag_trace_params": s.TraceParams,
             "svdag_server_config": s.ServerConfig, "svdag_request_result": s.RequestResult,
             "svdag_replay_action": s.ReplayAction, "svdag_shade_params": s.ShadeParams, "svdag_tuning": s.Tuning,
             "svdag_stats": s.Stats, "svdag_table_stats": s.TableStats, "svdag_alt_tuning": s.AltTuning,
             "svdag_server_memory": s.ServerMemory}
    lines = ["#include <stddef.h>", '#include "svdag.h"']
    for cname, cls in pairs.items():
        lines.append(f'_Static_assert(sizeof({cname}) == {C.sizeof(cls)}, "size of {cname}");')
        for fname, *_ in cls._fields_:
            off = getattr(cls, fname).offset
            lines.append(f'_Static_assert(offsetof({cname}, {fname}) == {off}, "{cname}.{fname}");')
    lines.append(f'_Static_assert(sizeof(svdag_hit) == {s.HIT_DTYPE.itemsize}, "size of svdag_hit");')
    lines.append("typedef void (*any_fn)(void);")
    lines.append("any_fn const every_function[] = {" + ", ".join(f"(any_fn)&{f}" for f in s.EXPORTED) + "};")
    lines.append("int main(void) { return every_function[0] == 0; }")
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines) + "\n")
    inc = os.path.join(ROOT, "include")
    libdir = os.path.dirname(s.LIB_PATH)
    r = subprocess.run(["gcc", "-std=c11", "-pedantic", "-Wall", "-Werror", "-I", inc, str(src), "-L", libdir, "-lsvdag",
                        "-Wl,--unresolved-symbols=ignore-in-shared-libs", "-o", str(tmp_path / "abi")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
