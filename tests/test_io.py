"""DAG import and export on the host: BasicDAG conversion, item snapshots and both file formats.

BasicDAGs are built here from voxel grids (the reference's BasicDAG layout, basic_dag.h: root at
index 0, inner nodes [child mask | child indices], 64-bit leaves at level levels - 2). The library's
conversion is compared word for word with a restatement of create_dag_cpu without colour import
(my_gpu_hash_dag_factory.cpp:316-418), and the converted items are decoded back to the grid.
"""
import os

import numpy as np
import pytest


def child_offset(c):
    return ((c >> 2) & 1, (c >> 1) & 1, c & 1)


def leaf_bit(x, y, z):
    """Voxel index of (x, y, z) in a 4^3 leaf: coarse child in bits 5..3, fine child in bits 2..0."""
    coarse = ((x >> 1) << 2) | ((y >> 1) << 1) | (z >> 1)
    fine = ((x & 1) << 2) | ((y & 1) << 1) | (z & 1)
    return coarse * 8 + fine


def build_basic_dag(grid, levels):
    """BasicDAG words of a boolean grid of side 2^levels (content-deduplicated, root at index 0)."""
    LL = levels - 2
    data = [0] * 9  # the root's header and up to 8 child indices come first; unused words stay 0
    memo = {}

    def node(level, x0, y0, z0):
        side = 1 << (levels - level)
        sub = grid[x0:x0 + side, y0:y0 + side, z0:z0 + side]
        if not sub.any():
            return None
        if level == LL:
            m = 0
            for x, y, z in zip(*np.nonzero(sub)):
                m |= 1 << leaf_bit(int(x), int(y), int(z))
            key = (level, m)
            if key not in memo:
                memo[key] = len(data)
                data.extend([m & 0xFFFFFFFF, m >> 32])
            return memo[key]
        h = side // 2
        kids = []
        mask = 0
        for c in range(8):
            dx, dy, dz = child_offset(c)
            k = node(level + 1, x0 + dx * h, y0 + dy * h, z0 + dz * h)
            if k is not None:
                mask |= 1 << c
                kids.append(k)
        key = (level, mask, tuple(kids))
        if level == 0:
            data[0:1 + len(kids)] = [mask] + kids
            return 0
        if key not in memo:
            memo[key] = len(data)
            data.extend([mask] + kids)
        return memo[key]

    assert node(0, 0, 0, 0) == 0
    return np.array(data, dtype=np.uint32)


def convert(data, levels, material):
    """create_dag_cpu without colour import, restated: post-order, memoised by BasicDAG index."""
    LL = levels - 2
    words = [[] for _ in range(levels - 1)]
    count = [0] * (levels - 1)
    memo = [{} for _ in range(levels - 1)]

    def visit(level, idx):
        if idx in memo[level]:
            return memo[level][idx]
        if level == LL:
            lo, hi = int(data[idx]), int(data[idx + 1])
            v = bin(lo).count("1") + bin(hi).count("1")
            w = [lo, hi]
            for nib in range(0, v, 8):
                k = min(8, v - nib)
                w.append((material * 0x11111111) & ((1 << (4 * k)) - 1))
            fill = material if lo == hi == 0xFFFFFFFF else None
        else:
            mask = int(data[idx]) & 0xFF
            kids, fills = [], []
            j = 0
            for c in range(8):
                if mask >> c & 1:
                    o, f = visit(level + 1, int(data[idx + 1 + j]))
                    kids.append(o)
                    fills.append(f)
                    j += 1
            uniform = mask == 0xFF and fills[0] is not None and all(f == fills[0] for f in fills)
            fill = fills[0] if uniform else None
            w = [(0xFF | (1 << 8) | (fill << 9)) if uniform else mask] + kids
        res = (count[level], fill)
        count[level] += 1
        words[level].extend(w)
        memo[level][idx] = res
        return res

    visit(0, 0)
    return words, count


def decode(snap, levels, xyz):
    """Material of each voxel through an item snapshot (None for empty)."""
    LL = levels - 2
    items = []
    at = 0
    for level in range(levels - 1):
        n, lst, w = int(snap.level_items[level]), [], snap.words[at:at + int(snap.level_words[level])]
        i = 0
        while i < len(w):
            if level == LL:
                v = bin(int(w[i])).count("1") + bin(int(w[i + 1])).count("1")
                k = 2 + (4 * v + 31) // 32
            else:
                k = 1 + bin(int(w[i]) & 0xFF).count("1")
            lst.append([int(v) for v in w[i:i + k]])
            i += k
        assert len(lst) == n
        items.append(lst)
        at += int(snap.level_words[level])
    out = []
    for x, y, z in xyz:
        o, res = 0, None
        for level in range(LL):
            s = levels - level - 1
            c = (((x >> s) & 1) << 2) | (((y >> s) & 1) << 1) | ((z >> s) & 1)
            it = items[level][o]
            if not (it[0] >> c) & 1:
                break
            o = it[1 + bin(it[0] & 0xFF & ((1 << c) - 1)).count("1")]
        else:
            it = items[LL][o]
            b = leaf_bit(x & 3, y & 3, z & 3)
            m = it[0] | (it[1] << 32)
            if (m >> b) & 1:
                r = bin(m & ((1 << b) - 1)).count("1")
                res = (it[2 + (r * 4) // 32] >> ((r * 4) % 32)) & 0xF
        out.append(res)
    return out


def random_grid(rng, levels):
    g = 1 << levels
    x, y, z = np.meshgrid(*(np.arange(g),) * 3, indexing="ij")
    grid = y < (g // 2 + (np.sin(x / 3.0) * 3).astype(int))
    for _ in range(4):
        c = rng.integers(0, g, 3)
        r = rng.integers(3, g // 3)
        grid |= (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= r * r
    grid &= rng.random(grid.shape) > 0.02  # some ragged leaves
    return grid


@pytest.mark.parametrize("levels,seed", [(4, 0), (5, 1), (6, 2)])
def test_basic_dag_conversion_matches_restatement_and_grid(svdag_lib, levels, seed):
    rng = np.random.default_rng(seed)
    grid = random_grid(rng, levels)
    data = build_basic_dag(grid, levels)
    snap = svdag_lib.basic_dag_to_items(data, levels, material=5)
    words, count = convert(data, levels, 5)
    assert [int(v) for v in snap.level_items] == count
    assert [int(v) for v in snap.level_words] == [len(w) for w in words]
    assert snap.words.tolist() == [v for w in words for v in w]
    g = 1 << levels
    xyz = [tuple(int(v) for v in rng.integers(0, g, 3)) for _ in range(3000)]
    got = decode(snap, levels, xyz)
    assert got == [5 if grid[p] else None for p in xyz]


def test_full_subtrees_get_fully_filled_headers(svdag_lib):
    levels = 5
    grid = np.zeros((32, 32, 32), bool)
    grid[:, :16, :] = True  # the lower half is solid: level-1 children at y=0 are fully filled
    snap = svdag_lib.basic_dag_to_items(build_basic_dag(grid, levels), levels, material=3)
    # the root has only the children of the solid lower half (y bit of the child index 0)
    assert int(snap.words[0]) == 0x33 and int(snap.level_items[0]) == 1
    lvl1 = snap.words[int(snap.level_words[0]):int(snap.level_words[0] + snap.level_words[1])]
    heads = {int(v) for v in lvl1 if int(v) & 0xFF == 0xFF and int(v) >> 8}
    assert heads == {0xFF | (1 << 8) | (3 << 9)}  # the solid level-1 node, fully filled with material 3


@pytest.mark.parametrize("bad", ["index", "empty_leaf", "empty_node", "material"])
def test_conversion_rejects_bad_input(svdag_lib, bad):
    import ctypes as C

    levels = 4
    data = build_basic_dag(random_grid(np.random.default_rng(3), levels), levels)
    material = 1
    if bad == "index":
        data = data.copy()
        data[1] = len(data) + 5
    elif bad == "empty_leaf":
        data = np.array([1, 2, 1, 4, 0, 0], np.uint32)  # root -> level-1 node -> leaf with no voxels
    elif bad == "empty_node":
        data = np.array([1, 2, 0], np.uint32)  # root -> level-1 node with no children
    else:
        material = 16
    L = svdag_lib.lib()
    lw, li, total = np.zeros(levels - 1, np.uint64), np.zeros(levels - 1, np.uint64), C.c_uint64()
    st = L.svdag_basic_dag_to_items(data.ctypes.data, len(data), levels, material, None, 0, lw.ctypes.data, li.ctypes.data,
                                    C.byref(total))
    assert st == (1 if bad == "material" else 4)


def test_file_formats_round_trip(svdag_lib, tmp_path):
    levels = 5
    data = build_basic_dag(random_grid(np.random.default_rng(4), levels), levels)
    f = svdag_lib.BasicDAGFile((-1.0, -2.0, -3.0), (1.0, 2.0, 3.0), levels, data)
    p = os.path.join(tmp_path, "scene.basic_dag")
    f.write(p)
    assert os.path.getsize(p) == 48 + 4 + 8 + 4 * len(data)
    g = svdag_lib.BasicDAGFile.read(p)
    assert g.bounds_min == (-1.0, -2.0, -3.0) and g.bounds_max == (1.0, 2.0, 3.0) and g.levels == levels
    assert np.array_equal(g.data, data)
    snap = svdag_lib.basic_dag_to_items(data, levels, 2)
    q = os.path.join(tmp_path, "scene.items")
    snap.write(q)
    back = svdag_lib.ItemSnapshot.read(q)
    assert back.levels == levels and np.array_equal(back.words, snap.words)
    assert np.array_equal(back.level_words, snap.level_words) and np.array_equal(back.level_items, snap.level_items)
    with open(q, "r+b") as fh:
        fh.write(b"XXXXXXXX")
    with pytest.raises(svdag_lib.SvdagError):
        svdag_lib.ItemSnapshot.read(q)
