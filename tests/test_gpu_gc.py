"""Garbage collection, the slab free list and memory reclamation in the serving loop.

MyGPUHashDAG::garbageCollect (my_gpu_hash_dag.cu:373-463) marks what the active roots reach;
freeInactiveItems (gpu_hash_table_base.cu:265-374) clears the rest and hands empty overflow slabs
back to the slab allocator (DynamicSlabAllocator::free, dynamic_slab_alloc.h:187-208). Here those
slabs go on per-size-class free lists that later overflow allocations pop. Every check compares the
DAG with the oracle canonically (or with itself before and after, where nothing may change).
"""
import os

import numpy as np
import pytest

from gpu_util import TERRAIN, gpu_canon, gpu_trace, sphere_edits, to_oracle_edit, to_svdag_edit

pytestmark = pytest.mark.gpu

LEVELS = 10
SCENE = dict(seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70, num_structures=24,
             structure_seed=5)


def edits_of(svdag_lib, oracle_mod, n, seed, rmax=40, near=32):
    raw = sphere_edits(oracle_mod, LEVELS, n, seed, rmin=6, rmax=rmax, near=near)
    return ([to_svdag_edit(svdag_lib, *e) for e in raw], [to_oracle_edit(oracle_mod, *e) for e in raw])


def test_gc_returns_empty_overflow_slabs_and_reuses_them(svdag_lib, oracle_mod):
    """Tables filled to 24 items per bucket (a full bucket slab) put every new item of the edits in
    overflow slabs. Undoing the edits and collecting frees those items, unlinks the slabs they leave
    empty and counts them out of the region in use; doing the edits again takes the slabs back from
    the free lists instead of growing the region, and both states equal the oracle's."""
    g = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=1 << 30, load_factor=24, undo_depth=64)
    g.build_terrain(**TERRAIN)
    o = oracle_mod.OracleDag(LEVELS)
    o.build_terrain(oracle_mod.TerrainParams(**TERRAIN))
    scene = o.canon()
    ge, oe = edits_of(svdag_lib, oracle_mod, 40, seed=71)
    used0 = g.stats().item_region_used_bytes
    for e in ge:
        g.edit(e)
    g.sync()
    used1 = g.stats().item_region_used_bytes
    assert used1 > used0
    for _ in ge:
        g.undo()
    assert gpu_canon(oracle_mod, g) == scene
    g.garbage_collect()
    st = g.stats()
    assert st.gc_freed_items > 0 and st.gc_freed_slabs > 0
    assert st.free_list_slabs >= st.gc_freed_slabs and st.free_list_bytes > 0
    assert st.item_region_used_bytes < used1  # empty overflow slabs count as free again
    assert gpu_canon(oracle_mod, g) == scene
    for a, b in zip(ge, oe):
        g.edit(a)
        o.edit(b)
    g.sync()
    st2 = g.stats()
    assert st2.free_list_slabs < st.free_list_slabs  # popped by the overflow allocations
    assert st2.item_region_used_bytes <= used1 * 1.01
    assert gpu_canon(oracle_mod, g) == o.canon()
    g.free()


def test_gc_keep_history_keeps_every_undo_state(svdag_lib, oracle_mod):
    """svdag_gc_keep_history marks from the current root and every undo and redo root: undo and
    redo then give back the same roots, the oldest, current and newest states equal the oracle's,
    and only garbage older than the history is freed. Every edit is centred on the surface, so each
    one changes the DAG and pushes one undo frame."""
    g = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=1 << 30, undo_depth=8)
    g.build_terrain(**TERRAIN)
    o = oracle_mod.OracleDag(LEVELS)
    o.build_terrain(oracle_mod.TerrainParams(**TERRAIN))
    ge, oe = edits_of(svdag_lib, oracle_mod, 14, seed=72, near=0)
    roots, states = [g.get_first_node_index()], {}
    for i, (a, b) in enumerate(zip(ge, oe)):
        g.edit(a)
        o.edit(b)
        roots.append(g.get_first_node_index())
        if i + 1 in (6, 12, 14):
            states[i + 1] = o.canon()
    assert len(set(roots)) == len(roots)
    # two undos: the history holds the 6 roots before them and the 2 undone ones
    g.undo()
    g.undo()
    assert g.stats().undo_count == 6 and g.stats().redo_count == 2
    g.garbage_collect(keep_history=True)
    st = g.stats()
    assert st.gc_freed_items > 0  # the states older than the 8-deep history are gone
    assert st.undo_count == 6 and st.redo_count == 2
    assert g.get_first_node_index() == roots[12]
    assert gpu_canon(oracle_mod, g) == states[12]
    for k in range(6):
        g.undo()
        assert g.get_first_node_index() == roots[11 - k]
    assert gpu_canon(oracle_mod, g) == states[6]
    for k in range(8):
        g.redo()
        assert g.get_first_node_index() == roots[7 + k]
    assert gpu_canon(oracle_mod, g) == states[14]
    g.free()


def test_gc_mark_overflow_frees_nothing(svdag_lib, oracle_mod):
    """When a level's frontier does not fit the scratch arena the collection returns SVDAG_ERR_OOM
    before its sweep: the DAG, a traced frame and the undo history are unchanged. The frontier limit
    is lowered through SVDAG_GC_MAX_FRONTIER so that a small scene reaches it."""
    g = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=1 << 30)
    g.build_terrain(**TERRAIN)
    ge, _ = edits_of(svdag_lib, oracle_mod, 6, seed=73)
    for e in ge:
        g.edit(e)
    g.sync()
    st = g.stats()
    assert max(st.level_items[: LEVELS - 1]) > 2048
    p = svdag_lib.get_trace_params((512.0, 900.0, 512.0), (512.0, 512.0, 512.0), 256, 256)
    before_frame = gpu_trace(svdag_lib, g, p)
    before = gpu_canon(oracle_mod, g)
    items = [g.table(l).stats().items for l in range(LEVELS - 1)]
    root = g.get_first_node_index()
    os.environ["SVDAG_GC_MAX_FRONTIER"] = "1024"
    try:
        with pytest.raises(svdag_lib.SvdagError) as err:
            g.garbage_collect()
        assert err.value.status == 2  # SVDAG_ERR_OOM
    finally:
        del os.environ["SVDAG_GC_MAX_FRONTIER"]
    assert [g.table(l).stats().items for l in range(LEVELS - 1)] == items  # nothing swept
    assert g.get_first_node_index() == root
    assert g.stats().undo_count == st.undo_count
    assert gpu_canon(oracle_mod, g) == before
    assert gpu_trace(svdag_lib, g, p).tobytes() == before_frame.tobytes()
    g.sync()
    # without the limit the same collection succeeds and keeps the reachable DAG
    g.garbage_collect()
    assert gpu_canon(oracle_mod, g) == before
    g.free()


def c4_long(svdag_lib, n_edits, rate, seed):
    import svdag.workloads as w

    duration = n_edits / rate
    times, edits, frames = w.c4_stream(rate, duration, seed=seed, levels=LEVELS, terrain=SCENE, rmax=48.0, copy_offset=64)
    return times, edits, frames


def to_oracle(oracle_mod, e):
    o = oracle_mod.Edit()
    o.tool, o.material, o.radius = e.tool, e.material, e.radius
    o.center[:], o.src[:], o.dst[:] = list(e.center), list(e.src), list(e.dst)
    o.noise_seed, o.noise_cell_log2 = e.noise_seed, e.noise_cell_log2
    return o


@pytest.mark.parametrize("plain", [False, True])
def test_long_served_stream_reclaims_memory(svdag_lib, oracle_mod, plain):
    """A served stream of 30 000 edits (3 000 through the plain loop) under a memory cap a few tens
    of MB above the scene: the loop collects garbage several times (keeping the undo history),
    rejects nothing, every edit succeeds and the final DAG equals the oracle's after the same edits
    one at a time."""
    n = 3000 if plain else 30000
    times, edits, frames = c4_long(svdag_lib, n, rate=20000.0, seed=17)
    assert len(edits) > 0.9 * n
    g = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=1 << 30, undo_depth=32)
    g.build_terrain(**SCENE)
    used0 = g.stats().item_region_used_bytes
    cam = svdag_lib.get_trace_params((512.0, 950.0, 150.0), (512.0, 550.0, 512.0), 320, 180)
    mib = 1 << 20
    with svdag_lib.Server(g, cam, max_batch=128, plain=plain, memory_cap_bytes=used0 + 96 * mib,
                          gc_threshold_bytes=used0 + (4 if plain else 16) * mib) as srv:
        res = srv.replay(edits, times, frames)
        mem = srv.memory()
    k = len(edits)
    bad = np.nonzero(res["status"][:k] != 0)[0]
    assert len(bad) == 0, f"edit {bad[0]} failed with status {res['status'][bad[0]]}"
    assert mem["rejected_edits"] == 0 and mem["failed_edits"] == 0
    assert mem["gc_runs"] >= 2, mem
    assert mem["gc_freed_bytes"] > 0
    assert mem["used_bytes"] <= used0 + 96 * mib
    assert g.get_first_node_index() == int(res["root_after"][k - 1])
    assert g.stats().undo_count == 32  # the history survived the collections
    o = oracle_mod.OracleDag(LEVELS)
    o.build_terrain(oracle_mod.TerrainParams(**SCENE))
    for e in edits:
        o.edit(to_oracle(oracle_mod, e))
    assert gpu_canon(oracle_mod, g) == o.canon()
    g.free()


def test_serving_loop_rejects_an_edit_that_cannot_fit(svdag_lib, oracle_mod):
    """Admission never launches an edit whose reserve exceeds the room left after a collection: it
    fails with SVDAG_ERR_OOM up front (counted as rejected), the DAG is left as it was, and the edits
    around it are served. With collection switched off the same holds without a collection."""
    for gc in (True, False):
        g = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=1 << 30)
        g.build_terrain(**SCENE)
        used0 = g.stats().item_region_used_bytes
        cam = svdag_lib.get_trace_params((512.0, 950.0, 150.0), (512.0, 550.0, 512.0), 160, 90)
        L = oracle_mod.lib()
        p = oracle_mod.TerrainParams(**SCENE)
        h = L.oracle_terrain_height(p, LEVELS, 300, 300)
        small = to_svdag_edit(svdag_lib, 0, 3, (300.0, float(h), 300.0), 6.0)
        huge = to_svdag_edit(svdag_lib, 0, 5, (512.0, 512.0, 512.0), 2000.0)  # reserve of gigabytes
        with svdag_lib.Server(g, cam, memory_cap_bytes=used0 + (64 << 20), gc=gc) as srv:
            t1 = srv.submit_edit(small)
            r1 = srv.poll(t1)
            root1 = r1.root_after
            t2 = srv.submit_edit(huge)
            r2 = srv.poll(t2)
            t3 = srv.submit_edit(to_svdag_edit(svdag_lib, 1, 0, (300.0, float(h), 300.0), 6.0))
            r3 = srv.poll(t3)
            mem = srv.memory()
        assert r1.status == 0 and r3.status == 0
        assert r2.status == 2  # SVDAG_ERR_OOM, before launch
        assert mem["rejected_edits"] == 1 and mem["failed_edits"] == 0
        assert (mem["gc_runs"] >= 1) == gc
        assert r3.root_after != root1
        o = oracle_mod.OracleDag(LEVELS)
        o.build_terrain(oracle_mod.TerrainParams(**SCENE))
        o.edit(to_oracle(oracle_mod, small))
        o.edit(to_oracle(oracle_mod, to_svdag_edit(svdag_lib, 1, 0, (300.0, float(h), 300.0), 6.0)))
        assert gpu_canon(oracle_mod, g) == o.canon()  # the huge edit left no trace
        g.free()
