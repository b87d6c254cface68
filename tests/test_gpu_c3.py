"""The batched form on a scaled C3 workload: 256 edits of uneven footprint (sphere/box 50/50, radius
or half-side log-uniform up to 128 voxels, 40 % add / 40 % remove / 20 % paint, centres near the
surface) on a depth-12 scene with structures. The edits applied as one batch (svdag_edit_apply_many:
runs of small edits in the persistent kernel, the others through the per-tool CUDA graphs) and one
at a time must leave DAGs that are canonically equal to each other and to the oracle's after the
same edits, and every edit's record must report success.
"""
import pytest

from gpu_util import gpu_canon

pytestmark = pytest.mark.gpu

LEVELS = 12


def to_oracle(oracle_mod, e):
    o = oracle_mod.Edit()
    o.tool, o.material, o.radius = e.tool, e.material, e.radius
    o.center[:], o.src[:], o.dst[:] = list(e.center), list(e.src), list(e.dst)
    o.noise_seed, o.noise_cell_log2 = e.noise_seed, e.noise_cell_log2
    return o


def test_c3_batched_equals_plain_and_the_oracle(svdag_lib, oracle_mod):
    import svdag.workloads as w

    terrain = dict(w.C2_TERRAIN, num_structures=16)
    edits = w.c3_edits(levels=LEVELS, terrain=terrain, rmax=4096.0 * (1 << LEVELS) / 131072)
    assert len(edits) == 256

    batched = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=8 << 30, scratch_bytes=2 << 30, persistent=True)
    batched.build_terrain(**terrain)
    n = batched.edit_batch(edits)
    batched.sync()
    recs = batched.edit_records(n)
    assert all(r.status == 0 for r in recs)
    assert sum(1 for r in recs if r.root_after != r.root_before) > 200

    plain = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=8 << 30, scratch_bytes=2 << 30)
    plain.build_terrain(**terrain)
    for e in edits:
        plain.edit(e)
    plain.sync()

    o = oracle_mod.OracleDag(LEVELS)
    o.build_terrain(oracle_mod.TerrainParams(**terrain))
    for e in edits:
        assert o.edit(to_oracle(oracle_mod, e)).status == 0
    want = o.canon()
    assert gpu_canon(oracle_mod, batched) == want
    assert gpu_canon(oracle_mod, plain) == want
    batched.free()
    plain.free()
