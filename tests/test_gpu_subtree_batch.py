"""Groups of subtree edits in the batched form. Small edits whose footprints lie in pairwise disjoint
subtrees are built side by side, one block each (k_edit_subtrees). Then every edit's path from its
subtree to the root is rebuilt, one level for all edits at a time, each edit's version of a node
taking the latest earlier edit's child where that edit's path passes, and the roots, records and
undo frames are committed in submission order (k_edit_spines).

Against the same edits applied one at a time:
 - the DAG after the batch equals the oracle's;
 - every edit's record chains: its root_before is the previous edit's root_after;
 - undo steps back through the same DAGs as the per-edit path, edit by edit;
 - the tables store each distinct item once, as many items per level as the per-edit path stores, even
   when many blocks make equal items at once.
A batch that mixes groups with overlapping edits, a large edit and a copy is checked the same way.
"""
import numpy as np
import pytest

from gpu_util import TERRAIN, gpu_canon

pytestmark = pytest.mark.gpu

LEVELS = 11


def scattered(svdag, n, seed, overlap_every=0):
    """Small sphere/box add, remove and paint edits at random places on the surface; with
    overlap_every, every such edit lands on the previous one."""
    import svdag.workloads as w

    rng = np.random.default_rng(seed)
    g = 1 << LEVELS
    tools = [svdag.TOOL_SPHERE_ADD, svdag.TOOL_SPHERE_REMOVE, svdag.TOOL_SPHERE_PAINT, svdag.TOOL_BOX_ADD,
             svdag.TOOL_BOX_REMOVE]
    out, prev = [], None
    for i in range(n):
        if overlap_every and prev is not None and i % overlap_every == 0:
            c = tuple(v + 3.0 for v in prev)
        else:
            x, z = (int(v) for v in rng.integers(8, g - 8, 2))
            c = (float(x), float(w.scene_height(LEVELS, x, z, **TERRAIN) + int(rng.integers(-4, 5))), float(z))
        prev = c
        out.append(w.make_edit(tools[int(rng.integers(0, len(tools)))], int(rng.integers(0, 16)), c, float(rng.integers(2, 18))))
    return out


def to_oracle(oracle_mod, e):
    o = oracle_mod.Edit()
    o.tool, o.material, o.radius = e.tool, e.material, e.radius
    o.center[:], o.src[:], o.dst[:] = list(e.center), list(e.src), list(e.dst)
    o.noise_seed, o.noise_cell_log2 = e.noise_seed, e.noise_cell_log2
    return o


def run_both(svdag_lib, oracle_mod, edits):
    batched = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=4 << 30, scratch_bytes=1 << 30, persistent=True, undo_depth=64)
    batched.build_terrain(**TERRAIN)
    n = batched.edit_batch(edits)
    batched.sync()
    recs = batched.edit_records(n)
    o = oracle_mod.OracleDag(LEVELS)
    o.build_terrain(oracle_mod.TerrainParams(**TERRAIN))
    for e in edits:
        assert o.edit(to_oracle(oracle_mod, e)).status == 0
    return batched, recs, o


def stored_items(dag):
    """Per level: the number of stored items, and how many of them repeat another's words."""
    out = []
    for level in range(LEVELS - 1):
        _, words = dag.export_level(level)
        out.append((len(words), len(words) - len(np.unique(words, axis=0)) if len(words) else 0))
    return out


def test_disjoint_small_edits_equal_the_oracle_and_chain(svdag_lib, oracle_mod):
    edits = scattered(svdag_lib, 96, seed=11)
    batched, recs, o = run_both(svdag_lib, oracle_mod, edits)
    assert [r.status for r in recs] == [0] * len(edits)
    for a, b in zip(recs, recs[1:]):
        assert b.root_before == a.root_after
    assert recs[-1].root_after == batched.get_first_node_index()
    assert sum(1 for r in recs if r.root_after != r.root_before) > 60
    assert gpu_canon(oracle_mod, batched) == o.canon()
    # the tables hold each distinct item once, exactly the items the per-edit path stores
    plain = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=4 << 30, scratch_bytes=1 << 30, undo_depth=64)
    plain.build_terrain(**TERRAIN)
    for e in edits:
        plain.edit(e)
    plain.sync()
    got, want = stored_items(batched), stored_items(plain)
    assert all(dup == 0 for _, dup in got), got
    assert [n for n, _ in got] == [n for n, _ in want]
    batched.free()
    plain.free()


def test_equal_new_items_from_many_edits_are_stored_once(svdag_lib, oracle_mod):
    """Many edits of one tool and material in scattered places produce many equal leaves and nodes
    at the same time; each must be stored once."""
    import svdag.workloads as w

    rng = np.random.default_rng(14)
    g = 1 << LEVELS
    edits = []
    for _ in range(120):
        x, z = (int(v) for v in rng.integers(16, g - 16, 2))
        c = (float(x), float(w.scene_height(LEVELS, x, z, **TERRAIN) + 6), float(z))
        edits.append(w.make_edit(svdag_lib.TOOL_BOX_ADD, 5, c, 7.0))
    batched, recs, o = run_both(svdag_lib, oracle_mod, edits)
    assert all(r.status == 0 for r in recs)
    assert gpu_canon(oracle_mod, batched) == o.canon()
    assert all(dup == 0 for _, dup in stored_items(batched))
    batched.free()


def test_undo_steps_back_edit_by_edit(svdag_lib, oracle_mod):
    edits = scattered(svdag_lib, 24, seed=12)
    batched, recs, _ = run_both(svdag_lib, oracle_mod, edits)
    plain = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=4 << 30, scratch_bytes=1 << 30, undo_depth=64)
    plain.build_terrain(**TERRAIN)
    states = [gpu_canon(oracle_mod, plain)]
    for e in edits:
        plain.edit(e)
        plain.sync()
        states.append(gpu_canon(oracle_mod, plain))
    assert gpu_canon(oracle_mod, batched) == states[-1]
    for k in range(len(edits), len(edits) - 8, -1):
        batched.undo()
        batched.sync()
        assert gpu_canon(oracle_mod, batched) == states[k - 1], f"after undoing edit {k}"
    for k in range(len(edits) - 8, len(edits) - 4):
        batched.redo()
        batched.sync()
        assert gpu_canon(oracle_mod, batched) == states[k + 1]
    batched.free()
    plain.free()


def test_groups_mixed_with_overlaps_large_edits_and_copies(svdag_lib, oracle_mod):
    import svdag.workloads as w

    edits = scattered(svdag_lib, 60, seed=13, overlap_every=5)
    g = 1 << LEVELS
    h = w.scene_height(LEVELS, g // 2, g // 2, **TERRAIN)
    edits.insert(20, w.make_edit(svdag_lib.TOOL_SPHERE_REMOVE, 0, (g / 2, h, g / 2), 300.0))  # large: its own pass
    edits.insert(40, w.make_edit(svdag_lib.TOOL_COPY, 0, (g / 4, h, g / 4), 12.0, src=(g / 4, h, g / 4),
                                 dst=(g / 4 + 40, h, g / 4)))
    batched, recs, o = run_both(svdag_lib, oracle_mod, edits)
    assert all(r.status == 0 for r in recs)
    for a, b in zip(recs, recs[1:]):
        assert b.root_before == a.root_after
    assert gpu_canon(oracle_mod, batched) == o.canon()
    batched.free()
