"""Subtree edits on the host: the geometry that groups a batch's small edits
(gpu-svdag-editing_b200/csrc/svdag_subtree.h, compiled here from tests/subtree_host.cpp), checked
against the oracle.

The grouped form builds each edit's subtree against the DAG as the group found it. That equals the
edits' own passes because:
 - an edit changes no voxel outside its node's region;
 - edits whose nodes are disjoint commute: the DAG after them, in either order, is the same, item for
   item (canonical digests per level);
 - after each edit of a group, every child of every node on its path is what the latest edit of the
   group through that child left there, which is how the batch rebuilds all paths one level at a
   time (k_edit_spines).
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
LEVELS = 8
TERRAIN = dict(seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70)


@pytest.fixture(scope="module")
def geo(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    so = str(tmp_path_factory.mktemp("subtree") / "subtree_host.so")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", os.path.join(HERE, "subtree_host.cpp"), "-o", so])
    lib = C.CDLL(so)
    lib.subtree_node_of.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.c_void_p]
    lib.subtree_disjoint.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p]
    return lib


def footprint(tool, c, r):
    """The editor's footprint box as the library's make_editor forms it."""
    c = np.asarray(c, np.float32)
    if tool in (0, 1, 4):  # spheres: centre + 0.5, radius at least 0.1
        r = np.float32(max(r, 0.1))
        cc = c + np.float32(0.5)
        return cc - r, cc + r
    r = np.float32(r)
    return c - r, (c + np.float32(1.0)) if r == 0 else c + r


def node_of(geo, tool, c, r):
    lo, hi = footprint(tool, c, r)
    lo, hi = np.ascontiguousarray(lo, np.float32), np.ascontiguousarray(hi, np.float32)
    level, path = C.c_uint32(), np.zeros(3, np.uint32)
    if not geo.subtree_node_of(lo.ctypes.data, hi.ctypes.data, LEVELS, C.byref(level), path.ctypes.data):
        return None
    return level.value, path


def scene(oracle_mod):
    o = oracle_mod.OracleDag(LEVELS)
    o.build_terrain(oracle_mod.TerrainParams(**TERRAIN))
    return o


def edit(oracle_mod, tool, mat, c, r):
    e = oracle_mod.Edit()
    e.tool, e.material, e.radius = tool, mat, float(r)
    e.center[:] = [float(v) for v in c]
    return e


def random_edit(rng, g):
    return (int(rng.choice([0, 1, 2, 3, 4])), int(rng.integers(0, 16)),
            tuple(float(v) for v in rng.uniform(0, g, 3)), float(rng.integers(0, 24)))


def test_an_edit_changes_nothing_outside_its_node(geo, oracle_mod):
    """Every voxel the oracle's edit changes, within the node's region grown by 24 voxels, lies in the
    node's region."""
    rng = np.random.default_rng(5)
    g = 1 << LEVELS
    checked = 0
    for _ in range(60):
        tool, mat, c, r = random_edit(rng, g)
        s = node_of(geo, tool, c, r)
        if s is None:
            continue
        level, path = s
        side = 1 << (LEVELS - level)
        o = scene(oracle_mod)
        # the node's region grown by 24 voxels on every side (a wrong node would show right next to it)
        lo0 = np.maximum(path.astype(np.int64) * side - 24, 0)
        hi0 = np.minimum(path.astype(np.int64) * side + side + 24, g)
        x, y, z = np.meshgrid(*(np.arange(a, b) for a, b in zip(lo0, hi0)), indexing="ij")
        xyz = np.stack([x.ravel(), y.ravel(), z.ravel()], 1).astype(np.uint32)
        before = o.sample(xyz)
        assert o.edit(edit(oracle_mod, tool, mat, c, r)).status == 0
        after = o.sample(xyz)
        changed = xyz[before != after]
        lo = path.astype(np.int64) * side
        inside = np.all((changed >= lo) & (changed < lo + side), axis=1)
        assert inside.all(), (tool, c, r, level, path)
        checked += 1
    assert checked >= 30


def test_edits_in_disjoint_nodes_commute(geo, oracle_mod):
    rng = np.random.default_rng(6)
    g = 1 << LEVELS
    pairs = 0
    while pairs < 25:
        a, b = random_edit(rng, g), random_edit(rng, g)
        sa, sb = node_of(geo, a[0], a[2], a[3]), node_of(geo, b[0], b[2], b[3])
        if sa is None or sb is None:
            continue
        disjoint = bool(geo.subtree_disjoint(sa[0], sa[1].ctypes.data, sb[0], sb[1].ctypes.data))
        if not disjoint:
            continue
        ab, ba = scene(oracle_mod), scene(oracle_mod)
        for o, order in ((ab, (a, b)), (ba, (b, a))):
            for t, m, c, r in order:
                assert o.edit(edit(oracle_mod, t, m, c, r)).status == 0
        assert ab.canon() == ba.canon(), (a, b)
        pairs += 1


def test_disjointness_is_ancestry(geo):
    p = np.array([3, 5, 6], np.uint32)
    child = np.array([6, 10, 13], np.uint32)  # a child of p one level down
    other = np.array([8, 10, 13], np.uint32)  # a child of another level-3 node
    d = lambda la, pa, lb, pb: bool(geo.subtree_disjoint(la, pa.ctypes.data, lb, pb.ctypes.data))
    assert not d(3, p, 4, child) and not d(4, child, 3, p)
    assert not d(3, p, 3, p)
    assert d(3, p, 4, other) and d(4, child, 4, other)


def test_path_versions_follow_the_latest_edit_per_child(geo, oracle_mod):
    """The rule by which a group's paths are rebuilt one level for all edits at once: applied one
    after another, after edit k every child of every node on k's path is that child as the latest
    edit j <= k whose path passes through it left it, or as the group found it where none does.
    Checked by handle (the oracle stores each distinct item once) on groups of consecutive edits in
    one 64-voxel region whose nodes are pairwise disjoint, as the batch planner forms them."""
    rng = np.random.default_rng(7)
    g = 1 << LEVELS
    shared = groups = 0
    while groups < 6:
        base = rng.integers(0, g - 64, 3)
        group = []
        for _ in range(200):
            if len(group) == 10:
                break
            tool, mat = int(rng.choice([0, 1, 2, 3, 4])), int(rng.integers(0, 16))
            c = tuple(float(v) for v in base + rng.uniform(0, 64, 3))
            r = float(rng.integers(0, 7))
            s = node_of(geo, tool, c, r)
            if s is None or not all(geo.subtree_disjoint(s[0], s[1].ctypes.data, q[0], q[1].ctypes.data)
                                    for _, q in group):
                continue
            group.append(((tool, mat, c, r), s))
        if len(group) < 4:
            continue
        o = scene(oracle_mod)
        kids = [np.array([(b >> 2) & 1, (b >> 1) & 1, b & 1], np.uint32) for b in range(8)]
        watch = {(l + 1, tuple(int(v) for v in (p >> (lv - l)) * 2 + kid))
                 for _, (lv, p) in group for l in range(lv) for kid in kids}
        snap = lambda: {key: o.node_at(key[0], np.array(key[1], np.uint32)) for key in watch}
        states = [snap()]
        for (tool, mat, c, r), _ in group:
            assert o.edit(edit(oracle_mod, tool, mat, c, r)).status == 0
            states.append(snap())
        for k, (_, (lk, pk)) in enumerate(group):
            for l in range(lk):
                for kid in kids:
                    child = tuple(int(v) for v in (pk >> (lk - l)) * 2 + kid)
                    through = [j for j, (_, (lj, pj)) in enumerate(group[:k + 1])
                               if lj > l and tuple(int(v) for v in pj >> (lj - l - 1)) == child]
                    want = states[through[-1] + 1] if through else states[0]
                    assert states[k + 1][(l + 1, child)] == want[(l + 1, child)], (k, l, child)
                    shared += bool(through) and through[-1] != k
        groups += 1
    assert shared > 50  # children last changed by an earlier edit of the group, not by edit k
