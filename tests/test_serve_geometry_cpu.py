"""The serving loop's host geometry, compiled from its own header for the host
(tests/serve_geometry_host.cpp over svdag_serve_geometry.h): the admission estimate bounds the items
an edit adds (checked against the oracle's counts); edit_boxes gives exactly the boxes the CPU claim
tests use (tests/test_incremental_frames_cpu.py, tests/test_edit_boxes_cpu.py check those boxes
against the oracle); box_rows' rectangle holds every hit-buffer pixel whose ray meets the box, so
copying only those rows and columns of an incremental frame misses no changed pixel."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from test_incremental_frames_cpu import boxes_of, camera, meets, rays

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def frames(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    so = str(tmp_path_factory.mktemp("frames") / "serve_geometry_host.so")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", os.path.join(HERE, "serve_geometry_host.cpp"), "-o", so])
    lib = C.CDLL(so)
    lib.frames_edit_boxes.restype = C.c_uint32
    lib.frames_edit_boxes.argtypes = [C.c_void_p, C.c_void_p]
    lib.frames_box_rows.restype = C.c_int
    lib.frames_box_rows.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.frames_edit_reserve_bytes.restype = C.c_ulonglong
    lib.frames_edit_reserve_bytes.argtypes = [C.c_void_p, C.c_uint32]
    return lib


def random_edits(svdag_lib, rng, n, g):
    for _ in range(n):
        e = svdag_lib.Edit(tool=int(rng.integers(0, 9)), material=int(rng.integers(0, 16)))
        e.radius = float(rng.choice([0.0, 0.05, 0.5, 1.0, float(rng.uniform(0, 300))]))
        e.center[:] = [float(v) for v in rng.uniform(-10, g + 10, 3)]
        e.src[:] = [float(v) for v in rng.uniform(0, g, 3)]
        e.dst[:] = [float(v) for v in rng.uniform(0, g, 3)]
        yield e


def test_edit_boxes_are_the_claim_tests_boxes(svdag_lib, frames):
    rng = np.random.default_rng(17)
    out = np.zeros(12, np.float32)
    for e in random_edits(svdag_lib, rng, 3000, 1 << 12):
        n = frames.frames_edit_boxes(C.addressof(e), out.ctypes.data)
        want = boxes_of(e)
        assert n == len(want)
        for i, b in enumerate(want):
            assert np.array_equal(out[6 * i:6 * i + 6], b), (e.tool, list(e.center), e.radius)


@pytest.mark.parametrize("view", ["oblique", "down", "side", "random1", "random2", "random3", "random4"])
def test_box_rows_hold_every_pixel_whose_ray_meets_the_box(svdag_lib, oracle_mod, frames, view):
    g = float(1 << 10)
    eye, target = camera(view, g)
    p = oracle_mod.camera_params(eye, target, 60.0, 96, 72)
    tp = svdag_lib.TraceParams()
    C.memmove(C.addressof(tp), C.addressof(p), C.sizeof(tp))
    o, ivd = rays(p)
    rng = np.random.default_rng(sum(map(ord, view)))
    out = np.zeros(4, np.int64)
    covered = small = 0
    for _ in range(300):
        c = rng.uniform(0.2 * g, 0.8 * g, 3)
        c[1] = rng.uniform(0.2 * g, 0.7 * g)
        r = float(rng.uniform(1, 80))
        b = np.concatenate([c - r, c + r]).astype(np.float32)
        hit = meets(o, ivd, b)  # (H, W): pixel row y, column x
        if not frames.frames_box_rows(C.addressof(tp), b.ctypes.data, out.ctypes.data):
            continue  # a corner behind the camera: the server copies the whole frame
        row0, row1, col0, col1 = (int(v) for v in out)
        ys, xs = np.nonzero(hit)
        rows = p.height - 1 - ys  # buffer row H - 1 - y holds pixel row y
        assert np.all((rows >= row0) & (rows <= row1) & (xs >= col0) & (xs <= col1)), (view, list(b))
        covered += int(hit.any())
        small += int((row1 - row0 + 1) * (col1 - col0 + 1) < p.width * p.height // 4)
    assert covered > 50 and small > 50  # the rectangles do cut the copy down


@pytest.mark.parametrize("tool", range(9))
def test_admission_estimate_bounds_the_new_items(svdag_lib, oracle_mod, frames, tool):
    """edit_reserve_bytes (what the server reserves before admitting an edit) is at least 50 bytes
    per item the edit adds, for edits of every tool and radii from 1 to 120 voxels near the surface
    of a depth-10 terrain, one after another (the oracle's new-item counts)."""
    levels = 10
    terrain = dict(seed=7, octaves=5, num_materials=8, min_height_pct=35, max_height_pct=65)
    L = oracle_mod.lib()
    o = oracle_mod.OracleDag(levels)
    o.build_terrain(oracle_mod.TerrainParams(**terrain))
    rng = np.random.default_rng(900 + tool)
    g = 1 << levels
    tight = 0.0
    for _ in range(14):
        x, z = (int(v) for v in rng.integers(130, g - 130, 2))
        h = L.oracle_terrain_height(oracle_mod.TerrainParams(**terrain), levels, x, z)
        e = oracle_mod.Edit(tool=tool, material=int(rng.integers(0, 16)))
        e.radius = float(np.exp(rng.uniform(0, np.log(120))))
        e.center[:] = [float(x), float(h + rng.integers(-8, 9)), float(z)]
        if tool in (5, 7):
            e.src[:] = list(e.center)
            e.dst[:] = [e.center[0] + float(rng.integers(-100, 101)), e.center[1] + float(rng.integers(-20, 21)),
                        e.center[2] + float(rng.integers(-100, 101))]
        if tool == 6:
            e.noise_seed, e.noise_cell_log2 = int(rng.integers(1, 99)), int(rng.integers(0, 4))
        if tool == 8:
            e.noise_seed = int(rng.integers(12, 22))
        se = svdag_lib.Edit()
        C.memmove(C.addressof(se), C.addressof(e), C.sizeof(se))
        reserve = frames.frames_edit_reserve_bytes(C.addressof(se), levels)
        st = o.edit(e)
        assert st.status == 0
        assert 50 * st.new_items <= reserve, (tool, e.radius, st.new_items, reserve)
        tight = max(tight, 50 * st.new_items / reserve)
    assert tight > 0.0  # the edits did add items
