"""Parity of the CUDA edit pipeline, tracer and voxel sampling with the CPU oracle.

Structure is compared canonically after every step (per-level distinct-content counts, per-level
digests and the Merkle root of the whole DAG), voxels in seeded dense bricks, hits pixel by pixel.
"""
import numpy as np
import pytest

from gpu_util import (TERRAIN, compare_hits, gpu_canon, gpu_sample, gpu_trace, random_bricks, sphere_edits,
                      to_oracle_edit, to_svdag_edit)

pytestmark = pytest.mark.gpu


def make_pair(svdag_lib, oracle_mod, levels, terrain=TERRAIN, pool=2 << 30):
    g = svdag_lib.MyGPUHashDAG(levels, pool_bytes=pool)
    g.build_terrain(**terrain)
    o = oracle_mod.OracleDag(levels)
    o.build_terrain(oracle_mod.TerrainParams(**terrain))
    return g, o


@pytest.mark.parametrize("levels", [6, 8, 10])
def test_terrain_build_parity(svdag_lib, oracle_mod, levels):
    g, o = make_pair(svdag_lib, oracle_mod, levels)
    assert gpu_canon(oracle_mod, g) == o.canon()
    rng = np.random.default_rng(levels)
    xyz = random_bricks(rng, levels, 16, 16)
    assert np.array_equal(gpu_sample(g, xyz), o.sample(xyz))
    g.free()


def test_sphere_edit_stream_c0(svdag_lib, oracle_mod):
    """64 sphere edits on the depth-10 terrain, structure compared after every edit."""
    levels = 10
    g, o = make_pair(svdag_lib, oracle_mod, levels)
    for i, (tool, mat, c, r) in enumerate(sphere_edits(oracle_mod, levels, 64, seed=2024)):
        so = o.edit(to_oracle_edit(oracle_mod, tool, mat, c, r))
        g.edit(to_svdag_edit(svdag_lib, tool, mat, c, r))
        sg = g.last_edit_stats()
        assert sg.status == 0
        assert list(sg.svo_nodes) == list(so.svo_nodes), i
        assert sg.unique_items == so.unique_items, i
        assert sg.new_items == so.new_items, i
        assert sg.edited_voxels == so.edited_voxels, i
        if i % 8 == 7 or i < 4:
            assert gpu_canon(oracle_mod, g) == o.canon(), i
    assert gpu_canon(oracle_mod, g) == o.canon()
    rng = np.random.default_rng(9)
    xyz = random_bricks(rng, levels, 32, 32)
    assert np.array_equal(gpu_sample(g, xyz), o.sample(xyz))
    p = svdag_lib.get_trace_params((512.0, 900.0, 512.0), (512.0, 512.0, 512.0), 256, 256)
    po = oracle_mod.TraceParams()
    for f in ("camera", "ray_min", "ray_ddx", "ray_ddy"):
        getattr(po, f)[:] = list(getattr(p, f))
    po.width, po.height = p.width, p.height
    compare_hits(gpu_trace(svdag_lib, g, p), o.trace(po, threads=8))
    g.free()


TOOLS = [
    ("box_add", 2, 5, (100.0, 150.0, 90.0), 21.0, {}),
    ("box_remove", 3, 0, (128.0, 140.0, 128.0), 30.0, {}),
    ("box_add_aligned", 2, 7, (64.0, 64.0, 64.0), 32.0, {}),
    ("sphere_paint", 4, 11, (120.0, 130.0, 60.0), 25.0, {}),
    ("noise_paint", 6, 0, (128.0, 128.0, 128.0), 60.0, {"noise_seed": 3, "noise_cell_log2": 3}),
    ("copy", 5, 0, (60.0, 140.0, 60.0), 20.0, {"src": (60.0, 140.0, 60.0), "dst": (190.0, 150.0, 180.0)}),
    ("copy_overlap", 5, 0, (100.0, 130.0, 100.0), 24.0, {"src": (100.0, 130.0, 100.0), "dst": (111.0, 137.0, 95.0)}),
    ("move", 7, 0, (70.0, 120.0, 200.0), 16.0, {"src": (70.0, 120.0, 200.0), "dst": (80.0, 160.0, 170.0)}),
    ("sphere_add_tiny", 0, 9, (33.0, 150.0, 77.0), 0.05, {}),
    ("sphere_remove_everything", 1, 0, (128.0, 128.0, 128.0), 300.0, {}),
]


@pytest.mark.parametrize("name,tool,mat,center,radius,kw", TOOLS, ids=[t[0] for t in TOOLS])
def test_tool_parity(svdag_lib, oracle_mod, name, tool, mat, center, radius, kw):
    levels = 8
    g, o = make_pair(svdag_lib, oracle_mod, levels)
    for _ in range(2):  # apply twice: the second edit meets the first one's output
        o.edit(to_oracle_edit(oracle_mod, tool, mat, center, radius, **kw))
        g.edit(to_svdag_edit(svdag_lib, tool, mat, center, radius, **kw))
        g.sync()
        assert gpu_canon(oracle_mod, g) == o.canon()
    rng = np.random.default_rng(1)
    xyz = random_bricks(rng, levels, 24, 16)
    assert np.array_equal(gpu_sample(g, xyz), o.sample(xyz))
    g.free()


def test_undo_redo_gc(svdag_lib, oracle_mod):
    levels = 8
    g, o = make_pair(svdag_lib, oracle_mod, levels)
    edits = sphere_edits(oracle_mod, levels, 12, seed=5, rmin=3, rmax=20, near=8)
    for tool, mat, c, r in edits:
        o.edit(to_oracle_edit(oracle_mod, tool, mat, c, r))
        g.edit(to_svdag_edit(svdag_lib, tool, mat, c, r))
    for step in ["undo", "undo", "undo", "redo", "undo", "redo", "redo"]:
        getattr(o, step)()
        getattr(g, step)()
        assert gpu_canon(oracle_mod, g) == o.canon(), step
    st = g.stats()
    assert st.undo_count == o.undo_count() and st.redo_count == o.redo_count()
    before = g.stats().level_items
    o.gc()
    g.garbage_collect()
    assert gpu_canon(oracle_mod, g) == o.canon()
    st = g.stats()
    assert st.undo_count == 0 and st.redo_count == 0
    assert sum(st.level_items) <= sum(before)
    # editing after a collection reuses freed slots and stays exact
    tool, mat, c, r = edits[0]
    o.edit(to_oracle_edit(oracle_mod, tool, mat, c, r))
    g.edit(to_svdag_edit(svdag_lib, tool, mat, c, r))
    assert gpu_canon(oracle_mod, g) == o.canon()
    g.free()


def test_trace_misses_and_empty_dag(svdag_lib, oracle_mod):
    g = svdag_lib.MyGPUHashDAG(6, pool_bytes=1 << 28)
    o = oracle_mod.OracleDag(6)
    p = svdag_lib.get_trace_params((-20.0, 80.0, -20.0), (32.0, 20.0, 32.0), 64, 48)
    po = oracle_mod.TraceParams()
    for f in ("camera", "ray_min", "ray_ddx", "ray_ddy"):
        getattr(po, f)[:] = list(getattr(p, f))
    po.width, po.height = p.width, p.height
    h = gpu_trace(svdag_lib, g, p)
    assert not h["path"].any()
    g.build_terrain(**TERRAIN)
    o.build_terrain(oracle_mod.TerrainParams(**TERRAIN))
    compare_hits(gpu_trace(svdag_lib, g, p), o.trace(po))
    g.free()


def test_batched_form_equals_sequential(svdag_lib, oracle_mod):
    """One persistent launch over a mixed batch gives the same DAG as the oracle applying the same
    edits one by one, and per-edit records match the oracle's per-edit counters."""
    levels = 8
    g, o = make_pair(svdag_lib, oracle_mod, levels)
    rng = np.random.default_rng(77)
    batch, oracle_edits = [], []
    for i, (tool, mat, c, r) in enumerate(sphere_edits(oracle_mod, levels, 24, seed=13, rmin=2, rmax=24, near=10)):
        kind = i % 6
        kw = {}
        if kind == 2:
            tool = 2 if rng.integers(0, 2) else 3  # box add / remove
        elif kind == 3:
            tool = 4  # sphere paint
        elif kind == 4:
            tool, kw = 6, {"noise_seed": 5, "noise_cell_log2": 2}
        elif kind == 5:
            tool, kw = (5 if rng.integers(0, 2) else 7), {"src": c, "dst": (c[0] + 9.0, c[1] + 3.0, c[2] - 7.0)}
        batch.append(to_svdag_edit(svdag_lib, tool, mat, c, r, **kw))
        oracle_edits.append(to_oracle_edit(oracle_mod, tool, mat, c, r, **kw))
    nrec = g.edit_batch(batch)
    recs = g.edit_records(nrec)
    ri = 0
    for e in oracle_edits:
        if e.tool == 7:  # a move is a removal then a paste: compare the final DAG only
            o.edit(e)
            ri += 2
            continue
        st = o.edit(e)
        assert recs[ri].status == 0
        assert recs[ri].edited_voxels == st.edited_voxels, ri
        assert recs[ri].new_items == st.new_items, ri
        assert recs[ri].unique_items == st.unique_items, ri
        assert recs[ri].svo_items == sum(st.svo_nodes), ri
        ri += 1
    assert ri == nrec
    g.sync()
    assert gpu_canon(oracle_mod, g) == o.canon()
    # the undo history holds one frame per edit (two per move), as with single calls
    g.undo()
    o.undo()
    assert gpu_canon(oracle_mod, g) == o.canon()
    g.free()
