"""Known-answer tests of the CPU oracle, mirroring the reference's own tests.

The reference ships no golden vectors for this path; its Catch2 tests check encodings and
brute-force voxel predicates. These tests restate them against the oracle (which is the checker of
the CUDA implementation): gpu_base_dag_test.cpp:5-95, gpu_hash_dag_tests.cpp:35-262.
"""
import math

import numpy as np
import pytest


@pytest.mark.parametrize("payload", [1, 2, 3, 4, 79, 90, 127, 255])
@pytest.mark.parametrize("mask", [1, 2, 3, 4, 79, 90, 127, 255])
def test_node_header_encoding(oracle_mod, payload, mask):
    # gpu_base_dag_test.cpp:5-21
    L = oracle_mod.lib()
    h = L.oracle_encode_node_header(mask, payload)
    assert L.oracle_header_child_mask(h) == mask
    assert L.oracle_header_user_payload(h) == payload
    assert (h & 0xFF) == mask  # Utils::child_mask


def _leaf_roundtrip(oracle_mod, mask, mats):
    L = oracle_mod.lib()
    buf = np.zeros(11, dtype=np.uint32)
    m = np.asarray(mats, dtype=np.uint32)
    size = L.oracle_build_leaf(mask, m.ctypes.data, buf.ctypes.data)
    assert 3 <= size <= 10
    assert buf[size] == 0 if size < 11 else True
    assert L.oracle_leaf_size(buf.ctypes.data) == size
    buf[size:10] = 0xFFFFFFFF  # words past the size must not matter
    import ctypes as C
    for i in range(64):
        out = C.c_uint32()
        filled = L.oracle_leaf_material(buf.ctypes.data, i, C.byref(out))
        if (mask >> i) & 1:
            assert filled and out.value == mats[i]
        else:
            assert not filled


@pytest.mark.parametrize("material", list(range(15)))
@pytest.mark.parametrize("mask", [0x1, 0xFFFFFFFFFFFFFFFF, 0xAAAAAAAAAAAAAAAA, 0xABABABABABABABAB])
def test_leaf_builder_fixed(oracle_mod, material, mask):
    # gpu_base_dag_test.cpp:29-62
    _leaf_roundtrip(oracle_mod, mask, [material] * 64)


def test_leaf_builder_varying(oracle_mod):
    # gpu_base_dag_test.cpp:64-94
    mask = sum(1 << i for i in range(64) if i % 3)
    _leaf_roundtrip(oracle_mod, mask, [i % 11 for i in range(64)])


def _cube(lo, hi):
    r = np.arange(lo, hi + 1, dtype=np.uint32)
    x, y, z = np.meshgrid(r, r, r, indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], 1)


@pytest.mark.parametrize("levels", [10, 17])
def test_create_box_in_dag(oracle_mod, levels):
    # gpu_hash_dag_tests.cpp:91-122: every voxel of the box +-1 through get_value
    d = oracle_mod.OracleDag(levels)
    d.build_box(100.0, 130.0, 0)
    xyz = _cube(99, 131)
    v = d.sample(xyz)
    inside = np.all((xyz >= 100) & (xyz < 130), axis=1)
    assert np.all(v[inside] == 0)
    assert np.all(v[~inside] == 0xFFFFFFFF)


def test_sphere_paint_overlap(oracle_mod):
    # gpu_hash_dag_tests.cpp:168-196
    e = oracle_mod.Edit(tool=4, material=13)
    center = (3599, 8440, 5045)
    e.center[:] = [float(c) for c in center]
    e.radius = 15.0
    L = oracle_mod.lib()
    rng = np.random.default_rng(5)
    pts = rng.integers(-15, 16, size=(4000, 3)) + np.array(center)
    import ctypes as C
    for p in pts:
        path = np.asarray(p, dtype=np.uint32)
        op = L.oracle_should_edit(C.byref(e), path.ctypes.data, 0, 1, 0, None)
        dist = math.sqrt(float(np.sum((np.array(center, dtype=np.float64) - p) ** 2)))
        if dist < 15 - 1:
            assert op != 3
        elif dist > 15 + 1:
            assert op == 3


def test_paint_sphere_inside_box(oracle_mod):
    # gpu_hash_dag_tests.cpp:198-262 (the reference runs the edit on the GPU; here the oracle does)
    d = oracle_mod.OracleDag(17)
    d.build_box(100.0, 130.0, 0)
    e = oracle_mod.Edit(tool=4, material=13)
    e.center[:] = [125.0, 115.0, 115.0]
    e.radius = 15.0
    d.edit(e)
    xyz = _cube(99, 131)
    v = d.sample(xyz)
    inside = np.all((xyz >= 100) & (xyz < 130), axis=1)
    assert np.all(v[~inside] == 0xFFFFFFFF)
    L = oracle_mod.lib()
    import ctypes as C
    for p, val in zip(xyz[inside][::7], v[inside][::7]):
        path = np.asarray(p, dtype=np.uint32)
        overlap = L.oracle_should_edit(C.byref(e), path.ctypes.data, 0, 1, 0, None) != 3
        assert val == (13 if overlap else 0)


TERRAIN = dict(seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70)


@pytest.fixture(scope="module")
def terrain8(oracle_mod):
    d = oracle_mod.OracleDag(8)
    d.build_terrain(oracle_mod.TerrainParams(**TERRAIN))
    return d


def test_terrain_voxels_match_heightfield(oracle_mod, terrain8):
    L = oracle_mod.lib()
    p = oracle_mod.TerrainParams(**TERRAIN)
    rng = np.random.default_rng(7)
    xyz = rng.integers(0, 256, size=(20000, 3)).astype(np.uint32)
    v = terrain8.sample(xyz)
    for (x, y, z), val in zip(xyz, v):
        h = L.oracle_terrain_height(p, 8, int(x), int(z))
        assert 0.40 * 256 - 1 <= h <= 0.70 * 256
        if y < h:
            assert val == (int(y) * 8) >> 8
        else:
            assert val == 0xFFFFFFFF


def test_undo_redo_restores_structure(oracle_mod):
    d = oracle_mod.OracleDag(8)
    d.build_terrain(oracle_mod.TerrainParams(**TERRAIN))
    c0 = d.canon()
    e = oracle_mod.Edit(tool=1, material=0)
    e.center[:] = [128.0, 100.0, 128.0]
    e.radius = 20.0
    d.edit(e)
    c1 = d.canon()
    assert c1["root"] != c0["root"]
    d.undo()
    assert d.canon() == c0
    d.redo()
    assert d.canon() == c1
    assert d.undo_count() == 1 and d.redo_count() == 0
    d.gc()
    assert d.canon() == c1 and d.undo_count() == 0


def test_edit_then_inverse_edit(oracle_mod):
    """Adding a sphere of the terrain's own material band then removing it leaves no voxels
    above the band; dedup keeps the DAG minimal (unique counts never exceed the SVO's)."""
    d = oracle_mod.OracleDag(8)
    d.build_terrain(oracle_mod.TerrainParams(**TERRAIN))
    e = oracle_mod.Edit(tool=0, material=3)
    e.center[:] = [60.0, 200.0, 60.0]
    e.radius = 9.0
    st = d.edit(e)
    assert st.unique_items <= sum(st.svo_nodes)
    xyz = _cube(55, 65)
    xyz[:, 1] += 140
    assert (d.sample(xyz) != 0xFFFFFFFF).any()
    e.tool = 1
    d.edit(e)
    assert (d.sample(xyz) == 0xFFFFFFFF).all()


def test_erosion_semantics(oracle_mod):
    """MyGpuSphereErosionEditor (my_gpu_dag_editors.h:538-589): threshold 25 keeps only voxels with all
    26 neighbours filled inside the sphere; threshold 0 removes an isolated voxel; voxels outside the
    sphere stay. A box of whole leaves builds no leaves and leaves the DAG unchanged
    (my_gpu_hash_dag_edits.cu:651), so the box is offset by one voxel."""
    import numpy as np

    o = oracle_mod.OracleDag(8)

    def edit(tool, center, radius, material=0, threshold=0):
        e = oracle_mod.Edit()
        e.tool, e.material, e.radius, e.noise_seed = tool, material, radius, threshold
        e.center[:] = list(center)
        assert o.edit(e).status == 0

    edit(2, (128.0, 128.0, 128.0), 60.0, 3)  # [68, 188)^3: leaf aligned
    assert o.root == 0xFFFFFFFF
    edit(2, (129.0, 129.0, 129.0), 60.0, 3)  # [69, 189)^3
    edit(2, (30.0, 30.0, 30.0), 0.0, 5)  # one voxel
    edit(8, (129.0, 160.0, 129.0), 40.0, threshold=25)
    edit(8, (30.0, 30.0, 30.0), 5.0, threshold=0)
    xyz = np.array([[129, 160, 129], [129, 188, 129], [71, 188, 71], [30, 30, 30]], dtype=np.uint32)
    assert o.sample(xyz).tolist() == [3, 0xFFFFFFFF, 3, 0xFFFFFFFF]
