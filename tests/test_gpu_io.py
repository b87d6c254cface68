"""DAG import and export on the GPU: item snapshots saved and loaded back, and BasicDAG geometry files
loaded as the reference's create_dag_cpu loads them without colour import, against the oracle."""
import os

import numpy as np
import pytest

from gpu_util import gpu_canon, gpu_sample, gpu_trace, random_bricks

pytestmark = pytest.mark.gpu

SCENE = dict(seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70, num_structures=16,
             structure_seed=7)


def snapshot_to_basic(snap):
    """BasicDAG words of a snapshot's geometry (root at index 0, leaves as their two mask words)."""
    levels = snap.levels
    LL = levels - 2
    items, at = [], 0
    for level in range(levels - 1):
        w, lst, i = snap.words[at:at + int(snap.level_words[level])], [], 0
        while i < len(w):
            if level == LL:
                v = bin(int(w[i])).count("1") + bin(int(w[i + 1])).count("1")
                k = 2 + (4 * v + 31) // 32
            else:
                k = 1 + bin(int(w[i]) & 0xFF).count("1")
            lst.append([int(x) for x in w[i:i + k]])
            i += k
        items.append(lst)
        at += int(snap.level_words[level])
    data, pos = [], {}

    def emit(level, o):
        if (level, o) in pos:
            return pos[(level, o)]
        it = items[level][o]
        idx = len(data)
        pos[(level, o)] = idx
        if level == LL:
            data.extend(it[:2])
        else:
            data.extend([it[0] & 0xFF] + [0] * (len(it) - 1))
            for j, c in enumerate(it[1:]):
                data[idx + 1 + j] = emit(level + 1, c)
        return idx

    assert emit(0, 0) == 0
    return np.array(data, dtype=np.uint32)


def test_snapshot_round_trip(svdag_lib, oracle_mod, tmp_path):
    levels = 10
    a = svdag_lib.MyGPUHashDAG(levels, pool_bytes=1 << 30)
    a.build_terrain(**SCENE)
    snap = a.save_items()
    assert int(snap.level_items[0]) == 1 and len(snap.words) == int(snap.level_words.sum())
    path = os.path.join(tmp_path, "scene.items")
    a.write_to(path)
    b = svdag_lib.MyGPUHashDAG(levels, pool_bytes=1 << 30)
    b.read_from(path)
    ca = gpu_canon(oracle_mod, a)
    assert gpu_canon(oracle_mod, b) == ca
    o = oracle_mod.OracleDag(levels)
    o.build_terrain(oracle_mod.TerrainParams(**SCENE))
    assert ca == o.canon()
    for level in range(levels - 1):  # reachable items plus the canonical fully-filled ones
        assert b.table(level).stats().items == a.table(level).stats().items, level
    assert b.stats().undo_count == 0
    # the loaded DAG edits and traces like the original
    p = svdag_lib.get_trace_params((512.0, 900.0, 512.0), (512.0, 512.0, 512.0), 128, 128)
    assert gpu_trace(svdag_lib, a, p).tobytes() == gpu_trace(svdag_lib, b, p).tobytes()
    import svdag.workloads as w

    e = w.make_edit(svdag_lib.TOOL_SPHERE_REMOVE, 0, (500.0, 600.0, 480.0), 40.0)
    a.edit(e)
    b.edit(e)
    assert gpu_canon(oracle_mod, b) == gpu_canon(oracle_mod, a)
    b.undo()
    assert gpu_canon(oracle_mod, b) == ca
    a.free()
    b.free()


def test_empty_and_invalid_snapshots(svdag_lib, oracle_mod):
    levels = 8
    g = svdag_lib.MyGPUHashDAG(levels, pool_bytes=256 << 20)
    empty = g.save_items()
    assert int(empty.level_items.sum()) == 0 and len(empty.words) == 0
    g.build_terrain(**SCENE)
    root = g.get_first_node_index()
    snap = g.save_items()
    bad = svdag_lib.ItemSnapshot(levels, snap.words.copy(), snap.level_words.copy(), snap.level_items.copy())
    bad.words[0] = int(bad.words[0]) & 0xFFFFFF00  # a root with no children
    bad2 = svdag_lib.ItemSnapshot(levels, snap.words.copy(), snap.level_words.copy(), snap.level_items.copy())
    bad2.words[1] = 0xFFFFFF  # a child ordinal out of range
    for b in (bad, bad2):
        with pytest.raises(svdag_lib.SvdagError) as ex:
            g.load_items(b)
        assert ex.value.status == 1
        assert g.get_first_node_index() == root  # rejected before anything changed
    g.load_items(empty)
    assert g.get_first_node_index() == 0xFFFFFFFF
    g.load_items(snap)
    o = oracle_mod.OracleDag(levels)
    o.build_terrain(oracle_mod.TerrainParams(**SCENE))
    assert gpu_canon(oracle_mod, g) == o.canon()
    g.free()


def test_basic_dag_file_loads_like_create_dag_cpu(svdag_lib, oracle_mod, tmp_path):
    """Geometry of a terrain written as a BasicDAG file and loaded with one material equals the
    oracle's terrain of one material band (every voxel material 0), canonically and voxel by voxel."""
    levels = 10
    terrain = dict(seed=3, octaves=5, num_materials=8, min_height_pct=35, max_height_pct=75)
    src = svdag_lib.MyGPUHashDAG(levels, pool_bytes=1 << 30)
    src.build_terrain(**terrain)
    data = snapshot_to_basic(src.save_items())
    f = svdag_lib.BasicDAGFile((0.0, 0.0, 0.0), (1024.0, 1024.0, 1024.0), levels, data)
    path = os.path.join(tmp_path, "terrain.basic_dag")
    f.write(path)
    g = svdag_lib.MyGPUHashDAG(levels, pool_bytes=1 << 30)
    hdr = g.load_basic_dag(path, material=0)
    assert hdr.bounds_max == (1024.0, 1024.0, 1024.0)
    o = oracle_mod.OracleDag(levels)
    o.build_terrain(oracle_mod.TerrainParams(**dict(terrain, num_materials=1)))
    assert gpu_canon(oracle_mod, g) == o.canon()
    rng = np.random.default_rng(11)
    xyz = random_bricks(rng, levels, 24, 16)
    got = gpu_sample(g, xyz)
    assert np.array_equal(got, o.sample(xyz))
    solid = gpu_sample(src, xyz) != 0xFFFFFFFF
    assert np.array_equal(got != 0xFFFFFFFF, solid) and (got[solid] == 0).all()
    src.free()
    g.free()
