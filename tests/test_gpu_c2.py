"""The at-scale sequence on the depth-17 scene (131072^3, 8 octaves, 4096 structures): a sphere carve
of radius 2048, a 512^3 copy-paste moved by (1024, 0, 0), a 1024^3 noise paint; then undo, redo and
garbage collection.

The oracle cannot hold the whole depth-17 DAG. Edits are local (a node's result depends only on its
own old content, the editor and, for a copy, the source box), so the oracle builds the scene clipped
to a box around each edit's footprint, applies the edit, and every level-9 node (256^3 voxels)
inside the box must equal the GPU's node canonically. Undo/redo must give back the exact roots, and
garbage collection must leave every reachable item (frames traced before and after are identical).
"""
import numpy as np
import pytest

from gpu_util import gpu_node_at, gpu_subtree_canon, gpu_trace

pytestmark = pytest.mark.gpu

LEVELS = 17
CMP_LEVEL = 9
SIDE = 1 << (LEVELS - CMP_LEVEL)


def align_box(lo, hi):
    lo = [int(np.floor(v / SIDE)) * SIDE for v in lo]
    hi = [int(np.ceil(v / SIDE)) * SIDE for v in hi]
    return lo, hi


def regions(edits):
    """One clipped box per edit, around a part of its footprint boundary near the surface."""
    carve, copy, paint = edits
    c, r = list(carve.center), carve.radius
    p = (c[0] + 0.7071 * r, c[1] - 0.7071 * r, c[2])  # on the carve shell, below the surface
    out = [align_box([v - 256 for v in p], [v + 256 for v in p])]
    src, dst, h = list(copy.src), list(copy.dst), copy.radius
    lo = [min(s, d) - h for s, d in zip(src, dst)]
    hi = [max(s, d) + h for s, d in zip(src, dst)]
    out.append(align_box(lo, hi))
    q, h = list(paint.center), paint.radius
    e = (q[0] + h, q[1], q[2])  # the box face at +x
    out.append(align_box([v - 256 for v in e], [v + 256 for v in e]))
    return out


def nodes_in(lo, hi):
    for x in range(lo[0] // SIDE, hi[0] // SIDE):
        for y in range(lo[1] // SIDE, hi[1] // SIDE):
            for z in range(lo[2] // SIDE, hi[2] // SIDE):
                yield (x, y, z)


def compare_region(oracle_mod, g, o, lo, hi):
    solid = 0
    for path in nodes_in(lo, hi):
        hg = gpu_node_at(g, CMP_LEVEL, path)
        ho = o.node_at(CMP_LEVEL, path)
        assert (hg is None) == (ho is None), path
        if hg is None:
            continue
        assert gpu_subtree_canon(oracle_mod, g, CMP_LEVEL, hg) == o.canon_at(CMP_LEVEL, ho), path
        solid += 1
    return solid


@pytest.fixture(scope="module")
def c2(svdag_lib, oracle_mod):
    import svdag.workloads as w

    g = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=56 << 30, scratch_bytes=16 << 30)
    g.build_terrain(**w.C2_TERRAIN)
    yield g, w.c2_edits(), oracle_mod.TerrainParams(**w.C2_TERRAIN)
    g.free()


def test_c2_sequence_regions_undo_redo_gc(svdag_lib, oracle_mod, c2):
    g, edits, params = c2
    boxes = regions(edits)
    roots = [g.get_first_node_index()]
    for e in edits:
        g.edit(e)
        st = g.last_edit_stats()
        assert st.status == 0
        assert st.edited_voxels > 0
        roots.append(g.get_first_node_index())
    assert len(set(roots)) == 4
    # Each edit against the oracle on its clipped box.
    oracles = []
    for e, (lo, hi) in zip(edits, boxes):
        o = oracle_mod.OracleDag(LEVELS)
        o.build_scene_region(params, lo, hi)
        oe = oracle_mod.Edit()
        oe.tool, oe.material, oe.radius = e.tool, e.material, e.radius
        oe.center[:], oe.src[:], oe.dst[:] = list(e.center), list(e.src), list(e.dst)
        oe.noise_seed, oe.noise_cell_log2 = e.noise_seed, e.noise_cell_log2
        assert o.edit(oe).status == 0
        assert compare_region(oracle_mod, g, o, lo, hi) > 0
        oracles.append(o)
    # Undo to the scene, redo to the end: the exact roots come back.
    for k in range(3):
        g.undo()
        assert g.get_first_node_index() == roots[2 - k]
    lo, hi = boxes[0]
    o = oracle_mod.OracleDag(LEVELS)
    o.build_scene_region(params, lo, hi)
    assert compare_region(oracle_mod, g, o, lo, hi) > 0  # the carve region before the carve
    for k in range(3):
        g.redo()
        assert g.get_first_node_index() == roots[1 + k]
    # GC (MyGPUHashDAGUndoRedo::garbageCollect) clears the history and frees everything the current
    # root does not reach: the items of the replaced scene parts go, every reachable item stays (a
    # 1080p frame is unchanged, the paint region still equals the oracle's), undo has nothing left.
    cam = (0.30 * (1 << LEVELS) + 3000.0, 0.62 * (1 << LEVELS), 0.30 * (1 << LEVELS) - 2500.0)
    p = svdag_lib.get_trace_params(cam, tuple(edits[0].center), 1920, 1080)
    before = gpu_trace(svdag_lib, g, p)
    used, free_before = g.stats().item_region_used_bytes, g.stats().free_list_bytes
    items = [g.table(l).stats().items for l in range(LEVELS - 1)]
    g.garbage_collect()
    after_items = [g.table(l).stats().items for l in range(LEVELS - 1)]
    assert sum(after_items) < sum(items)
    st = g.stats()
    # freed slots stay in their slabs for reuse; overflow slabs left empty go on the free lists and
    # count as free
    assert st.item_region_used_bytes == used - (st.free_list_bytes - free_before)
    assert st.gc_freed_items == sum(items) - sum(after_items)
    assert g.stats().undo_count == 0 and g.stats().redo_count == 0
    after = gpu_trace(svdag_lib, g, p)
    assert before.tobytes() == after.tobytes()
    assert (after["material"] != 255).mean() > 0.5
    lo, hi = boxes[2]
    assert compare_region(oracle_mod, g, oracles[2], lo, hi) > 0
    g.undo()
    assert g.get_first_node_index() == roots[3]


def test_c2_1080p_frame_equals_the_oracle_in_a_clipped_region(svdag_lib, oracle_mod, c2):
    """A 1920x1080 frame of the depth-17 scene, pixel for pixel against the oracle. The camera looks
    steeply down at the terrain away from the edited regions, and the oracle builds the scene clipped
    to a box around it that holds every voxel the frame's rays reach first: every ray hits inside the
    box (checked), so the clipped scene and the whole one give the same frame."""
    from gpu_util import compare_hits
    from oracle import oracle as om

    g, _, params = c2
    L = oracle_mod.lib()
    gsz = 1 << LEVELS
    x0, z0 = int(0.80 * gsz), int(0.20 * gsz)
    h0 = L.oracle_terrain_height(params, LEVELS, x0, z0)
    cam = (float(x0), float(h0 + 160), float(z0))
    target = (float(x0 + 110), float(h0 - 120), float(z0 + 80))
    p = svdag_lib.get_trace_params(cam, target, 1920, 1080)
    hits = gpu_trace(svdag_lib, g, p)
    lo = [x0 - 2048, h0 - 2048, z0 - 2048]
    hi = [x0 + 2048, h0 + 1024, z0 + 2048]
    o = oracle_mod.OracleDag(LEVELS)
    o.build_scene_region(params, lo, hi)
    po = oracle_mod.TraceParams()
    for f in ("camera", "ray_min", "ray_ddx", "ray_ddy"):
        getattr(po, f)[:] = list(getattr(p, f))
    po.width, po.height = p.width, p.height
    import os

    ref = o.trace(po, max(1, len(os.sched_getaffinity(0))))
    path = hits["path"].astype(np.int64)
    assert np.all(np.any(path != 0, axis=1)), "every ray hits the terrain"
    inside = np.all((path >= np.array(lo) + 1) & (path < np.array(hi) - 1), axis=1)
    assert inside.all(), "every hit lies inside the clipped box"
    compare_hits(hits, ref)
    assert len(np.unique(path, axis=0)) > 10000  # a real view: the rays reach many distinct voxels
    del om
