"""The changed-region boxes of incremental served frames hold every voxel an edit changes: for every
tool, voxels sampled densely around the edit (and around a copy's or move's destination) that differ
before and after the edit all lie inside one of the edit's boxes. Checked with the oracle."""
import numpy as np
import pytest

from test_incremental_frames_cpu import boxes_of

LEVELS = 8
SCENE = dict(seed=4, octaves=5, num_materials=8, min_height_pct=35, max_height_pct=65)


def region(center, r, margin=12):
    lo = np.maximum(np.floor(np.array(center) - r - margin).astype(int), 0)
    hi = np.minimum(np.ceil(np.array(center) + r + margin).astype(int) + 1, 1 << LEVELS)
    ax = [np.arange(lo[i], hi[i]) for i in range(3)]
    g = np.stack(np.meshgrid(*ax, indexing="ij"), -1).reshape(-1, 3)
    return g.astype(np.uint32)


@pytest.mark.parametrize("tool", [0, 1, 2, 3, 4, 5, 6, 7, 8])
def test_boxes_hold_every_changed_voxel(oracle_mod, tool):
    L = oracle_mod.lib()
    rng = np.random.default_rng(40 + tool)
    o = oracle_mod.OracleDag(LEVELS)
    o.build_terrain(oracle_mod.TerrainParams(**SCENE))
    g = 1 << LEVELS
    changed_total = 0
    for _ in range(6):
        x, z = (int(v) for v in rng.integers(16, g - 16, 2))
        h = L.oracle_terrain_height(oracle_mod.TerrainParams(**SCENE), LEVELS, x, z)
        e = oracle_mod.Edit()
        e.tool, e.material = tool, int(rng.integers(0, 16))
        e.radius = float(rng.integers(0, 14)) + (0.5 if rng.random() < 0.3 else 0.0)
        e.center[:] = [float(x), float(h + rng.integers(-4, 5)), float(z)]
        centers = [list(e.center)]
        if tool in (5, 7):
            e.src[:] = list(e.center)
            e.dst[:] = [e.center[0] + float(rng.integers(-30, 31)), e.center[1] + float(rng.integers(-5, 6)),
                        e.center[2] + float(rng.integers(-30, 31))]
            centers.append([e.dst[i] + (e.center[i] - e.src[i]) for i in range(3)])
        if tool == 6:
            e.noise_seed, e.noise_cell_log2 = int(rng.integers(1, 99)), int(rng.integers(0, 4))
        if tool == 8:
            e.noise_seed = int(rng.integers(4, 20))
        xyz = np.concatenate([region(c, e.radius) for c in centers])
        before = o.sample(xyz)
        assert o.edit(e).status == 0
        after = o.sample(xyz)
        diff = xyz[before != after].astype(np.float64)
        changed_total += len(diff)
        inside = np.zeros(len(diff), bool)
        for b in boxes_of(e):
            b = b.astype(np.float64)
            # a voxel is the unit cube [v, v + 1): it must lie within the box
            inside |= np.all((diff >= b[:3]) & (diff + 1 <= b[3:]), axis=1)
        assert inside.all(), (tool, list(e.center), e.radius, diff[~inside][:5])
    assert changed_total > 0
