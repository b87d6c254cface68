"""The CUDA library's DAG read and edited by the reference's own code (oracle/_ref).

The level tables the GPU holds are exported and handed to the reference's DAGUtils::get_value and
editors (oracle/ref_harness.cu). Checked on the GPU:
  - every sampled voxel of the GPU DAG decodes through the reference's get_value to the value the
    GPU's own sampling kernel returns (the item encoding is the reference's);
  - after an edit of every reference tool, the GPU DAG's voxels equal the reference editors'
    decisions evaluated voxel by voxel over the GPU DAG as it was before the edit.
Skipped where oracle/_ref was not built (no reference sources when the repository was prepared).
"""
import numpy as np
import pytest

from gpu_util import TERRAIN, gpu_sample, to_svdag_edit

pytestmark = pytest.mark.gpu

LEVELS = 10


@pytest.fixture(scope="module")
def ref_mod():
    from oracle import ref

    if ref.lib() is None:
        pytest.skip("oracle/_ref is not built")
    return ref


def gpu_ref_dag(ref_mod, dag):
    dumps = [dag.export_level(l) for l in range(LEVELS - 1)]
    return ref_mod.RefDag(LEVELS, ref_mod.items_from_dumps(LEVELS, dag.get_first_node_index(), dumps))


def surface(oracle_mod, rng, dy=0):
    L = oracle_mod.lib()
    p = oracle_mod.TerrainParams(**TERRAIN)
    x, z = (int(v) for v in rng.integers(16, (1 << LEVELS) - 16, 2))
    return np.array([x, L.oracle_terrain_height(p, LEVELS, x, z) + dy, z], dtype=np.float64)


CASES = [(0, 14.0), (1, 22.0), (2, 10.0), (3, 15.0), (4, 18.0), (5, 11.0), (8, 9.0), (1, 1.5), (0, 3.25)]


def test_gpu_edits_equal_the_reference_editors(svdag_lib, oracle_mod, ref_mod):
    rng = np.random.default_rng(515)
    g = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=1 << 30)
    g.build_terrain(**TERRAIN)
    for i, (tool, radius) in enumerate(CASES):
        before = gpu_ref_dag(ref_mod, g)
        c = surface(oracle_mod, rng) + (0.31 if i % 2 else 0.0)
        kw, lo, hi = {}, c - radius - 3, c + radius + 3
        if tool == 5:
            dst = c + np.array([float(rng.integers(-40, 41)), 12.0, float(rng.integers(-40, 41))])
            kw = dict(src=tuple(c), dst=tuple(dst))
            lo, hi = dst - radius - 3, dst + radius + 3
        if tool == 8:
            kw = dict(noise_seed=int(rng.integers(8, 18)))
        e = to_svdag_edit(svdag_lib, tool, int(rng.integers(0, 16)), tuple(c), radius, **kw)
        g.edit(e)
        g.sync()
        lo = np.clip(np.floor(lo).astype(np.int64), 0, (1 << LEVELS) - 1)
        hi = np.clip(np.ceil(hi).astype(np.int64), 0, (1 << LEVELS) - 1)
        axes = [np.arange(lo[a], hi[a] + 1) for a in range(3)]
        xyz = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3).astype(np.uint32)
        want = before.edit_values(e, xyz)
        got = gpu_sample(g, xyz)
        bad = np.nonzero(want != got)[0]
        assert len(bad) == 0, (i, tool, xyz[bad[:5]].tolist(), want[bad[:5]].tolist(), got[bad[:5]].tolist())
        # the GPU's own sampling and the reference's decoding of the exported tables agree everywhere
        after = gpu_ref_dag(ref_mod, g)
        pts = np.concatenate([xyz, rng.integers(0, 1 << LEVELS, (50000, 3)).astype(np.uint32)])
        assert np.array_equal(after.get_values(pts), gpu_sample(g, pts))
    g.free()
