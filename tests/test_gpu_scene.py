"""GPU scene construction: terrain plus structures, one pass and tiled, against the oracle.

The oracle builds the scene with its own restatement of the structure generator and a plainer
classification (any structure bounding box touching a node forces subdivision), so agreement checks
the GPU's cell lists and structure/node tests as well as the pipeline. At full depth the oracle
cannot hold the whole DAG: subtrees under sampled nodes near the surface are compared canonically,
and sampled voxel bricks are compared with the scene definition itself.
"""
import numpy as np
import pytest

from gpu_util import gpu_canon, gpu_node_at, gpu_sample, gpu_subtree_canon, random_bricks

pytestmark = pytest.mark.gpu

SCENE = dict(seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70, num_structures=16,
             structure_seed=7)


def surface_bricks(oracle_mod, params, levels, rng, n, size):
    """Voxel bricks centred on the terrain surface (where the structures are)."""
    L = oracle_mod.lib()
    g = 1 << levels
    out = []
    r = np.arange(size)
    x, y, z = np.meshgrid(r, r, r, indexing="ij")
    off = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    for _ in range(n):
        bx, bz = (int(v) for v in rng.integers(0, g - size, 2))
        h = L.oracle_terrain_height(params, levels, bx, bz)
        by = int(min(max(h - size // 2, 0), g - size))
        out.append(off + np.array([bx, by, bz]))
    return np.concatenate(out).astype(np.uint32)


@pytest.mark.parametrize("levels,tile_level", [(9, 0), (10, 0), (10, 2), (10, 4)])
def test_scene_with_structures_matches_oracle(svdag_lib, oracle_mod, levels, tile_level):
    p = oracle_mod.TerrainParams(**SCENE)
    o = oracle_mod.OracleDag(levels)
    o.build_terrain(p)
    g = svdag_lib.MyGPUHashDAG(levels, pool_bytes=2 << 30)
    g.build_terrain(**SCENE, tile_level=tile_level)
    assert gpu_canon(oracle_mod, g) == o.canon()
    rng = np.random.default_rng(levels + tile_level)
    xyz = surface_bricks(oracle_mod, p, levels, rng, 12, 16)
    got = gpu_sample(g, xyz)
    assert np.array_equal(got, o.sample(xyz))
    assert np.array_equal(got, oracle_mod.scene_voxels(p, levels, xyz))
    g.free()


def test_tiled_build_equals_one_pass_build(svdag_lib, oracle_mod):
    """The same scene built whole and cut into tiles gives the same DAG (canonically) and tables
    holding exactly the reachable items plus the canonical fully-filled ones."""
    levels = 11
    params = dict(SCENE, num_structures=48, structure_seed=3)
    a = svdag_lib.MyGPUHashDAG(levels, pool_bytes=4 << 30)
    a.build_terrain(**params)
    b = svdag_lib.MyGPUHashDAG(levels, pool_bytes=4 << 30)
    b.build_terrain(**params, tile_level=3)
    ca, cb = gpu_canon(oracle_mod, a), gpu_canon(oracle_mod, b)
    assert ca == cb
    for l in range(levels - 1):
        assert a.table(l).stats().items == b.table(l).stats().items, l
    a.free()
    b.free()


def c2_scene(levels):
    return dict(seed=0, octaves=8, num_materials=8, min_height_pct=40, max_height_pct=70, num_structures=4096,
                structure_seed=11)


@pytest.mark.parametrize("levels", [13])
def test_tiled_scene_subtrees_match_oracle(svdag_lib, oracle_mod, levels):
    """A tiled scene with the full structure count: subtrees under sampled level-(levels-7) nodes on
    the surface equal the oracle's builds of the same nodes; bricks equal the scene definition."""
    params = c2_scene(levels)
    p = oracle_mod.TerrainParams(**params)
    g = svdag_lib.MyGPUHashDAG(levels, pool_bytes=8 << 30)
    g.build_terrain(**params, tile_level=3)
    L = oracle_mod.lib()
    rng = np.random.default_rng(5)
    level = levels - 7
    checked = 0
    for _ in range(6):
        x, z = (int(v) for v in rng.integers(0, 1 << levels, 2))
        y = L.oracle_terrain_height(p, levels, x, z)
        path = (x >> (levels - level), y >> (levels - level), z >> (levels - level))
        h = gpu_node_at(g, level, path)
        o = oracle_mod.OracleDag(levels)
        ho = o.build_scene_subtree(p, level, path)
        assert (h is None) == (ho == 0xFFFFFFFF), path
        if h is None:
            continue
        assert gpu_subtree_canon(oracle_mod, g, level, h) == o.canon_at(level, ho), path
        checked += 1
    assert checked >= 3
    xyz = surface_bricks(oracle_mod, p, levels, rng, 16, 16)
    assert np.array_equal(gpu_sample(g, xyz), oracle_mod.scene_voxels(p, levels, xyz))
    g.free()
