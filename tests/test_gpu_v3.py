"""The reference's own DAG file (MyGPUHashDAG::writeTo / readFrom, version 3) against the reference's
own code: its host DAG MyGPUHashDAG<EMemoryType::CPU>, compiled from its sources into oracle/_ref
(oracle/ref_v3_harness.cu). That DAG copies its host arrays with cudaMemcpy, so these run where a
CUDA driver is, on the GPU box.

 - A file the reference writes (its DAG filled from an oracle DAG through find/add, resized by
   setLoadFactor, then writeTo) is read by the library's reader into the same DAG, and by the CUDA
   library's readFrom into a DAG canonically equal to the oracle's.
 - A file the library writes (from the oracle's snapshot, and from the CUDA library's DAG through
   writeTo) is read by the reference's readFrom into the same DAG; the reference's find locates
   every reachable item at its own handle, and its DAGUtils::get_value equals the oracle's voxels.
"""
import numpy as np
import pytest

from gpu_util import gpu_canon
from snapshot_util import same_dag, snap_parts, snapshot_from_rows

pytestmark = pytest.mark.gpu

EDITS = [  # tool, material, centre, radius: on an empty scene of the reference's depth
    (2, 7, (40000.0, 40000.0, 40000.0), 70.0),  # box add: fully-filled nodes
    (0, 3, (40060.0, 40010.0, 39990.0), 55.0),
    (4, 11, (40030.0, 40040.0, 40020.0), 30.0),  # paint
    (1, 0, (39990.0, 40000.0, 40050.0), 25.0),  # carve
    (0, 14, (90001.5, 12000.0, 65000.0), 20.0),  # a second, far island
]


@pytest.fixture(scope="module")
def ref_mod(oracle_mod):
    from oracle import ref

    if ref.lib() is None:
        pytest.skip("oracle/_ref is not built (the reference sources were absent where the tests were prepared)")
    return ref


def oracle_edit(oracle_mod, tool, mat, c, r):
    e = oracle_mod.Edit()
    e.tool, e.material, e.radius = tool, mat, r
    e.center[:] = list(c)
    return e


def gpu_edit(svdag, tool, mat, c, r):
    e = svdag.Edit()
    e.tool, e.material, e.radius = tool, mat, r
    e.center[:] = list(c)
    return e


@pytest.fixture(scope="module")
def scene(svdag_lib, oracle_mod, ref_mod):
    levels = ref_mod.v3_levels()
    o = oracle_mod.OracleDag(levels)
    for ed in EDITS:
        assert o.edit(oracle_edit(oracle_mod, *ed)).status == 0
    snap = snapshot_from_rows(svdag_lib, levels, o.export_items())
    rng = np.random.default_rng(7)
    near = np.concatenate([np.asarray(c) + rng.uniform(-1.3 * r, 1.3 * r, (1500, 3)) for _, _, c, r in EDITS])
    xyz = np.concatenate([near, rng.uniform(0, 1 << levels, (2000, 3))]).astype(np.uint32)
    return levels, o, snap, xyz


def test_the_library_reads_what_the_reference_writes(svdag_lib, oracle_mod, ref_mod, scene, tmp_path):
    levels, o, snap, _ = scene
    p = str(tmp_path / "ref.v3")
    ref_mod.v3_write(*snap_parts(snap), p)
    back = svdag_lib.v3_to_items(p, levels)
    assert same_dag(levels, snap_parts(snap), snap_parts(back))
    dag = svdag_lib.MyGPUHashDAG(levels, pool_bytes=2 << 30, scratch_bytes=512 << 20)
    dag.readFrom(p)
    assert gpu_canon(oracle_mod, dag) == o.canon()
    dag.free()


def test_the_reference_reads_what_the_library_writes(svdag_lib, ref_mod, scene, tmp_path):
    levels, o, snap, xyz = scene
    p = str(tmp_path / "lib.v3")
    svdag_lib.items_to_v3(snap, p, svdag_lib.V3_CPU)
    with ref_mod.RefV3Dag(p) as r:
        w, lw, li, found = r.items()
        assert same_dag(levels, (w, lw, li), snap_parts(snap))
        assert found == int(li.sum())
        got = r.get_values(xyz)
    assert np.array_equal(got, o.sample(xyz))
    assert (got != 0xFFFFFFFF).sum() > 1000


def test_cuda_dag_write_and_read_through_the_reference(svdag_lib, oracle_mod, ref_mod, scene, tmp_path):
    levels, o, snap, xyz = scene
    dag = svdag_lib.MyGPUHashDAG(levels, pool_bytes=2 << 30, scratch_bytes=512 << 20)
    dag.load_items(snap)
    extra = (0, 9, (40100.0, 39950.0, 40020.0), 33.0)
    dag.edit(gpu_edit(svdag_lib, *extra))
    dag.sync()
    o2 = oracle_mod.OracleDag(levels)
    for ed in EDITS + [extra]:
        assert o2.edit(oracle_edit(oracle_mod, *ed)).status == 0
    p = str(tmp_path / "cuda.v3")
    dag.writeTo(p, svdag_lib.V3_CPU)
    with ref_mod.RefV3Dag(p) as r:
        w, lw, li, found = r.items()
        assert found == int(li.sum())
        assert np.array_equal(r.get_values(xyz), o2.sample(xyz))
    want = snapshot_from_rows(svdag_lib, levels, o2.export_items())
    assert same_dag(levels, (w, lw, li), snap_parts(want))
    # and back into a fresh CUDA DAG
    again = svdag_lib.MyGPUHashDAG(levels, pool_bytes=2 << 30, scratch_bytes=512 << 20)
    again.readFrom(p)
    assert gpu_canon(oracle_mod, again) == o2.canon()
    dag.free()
    again.free()


def test_empty_dag_through_the_reference(svdag_lib, ref_mod, tmp_path):
    levels = ref_mod.v3_levels()
    nl = levels - 1
    empty = svdag_lib.ItemSnapshot(levels, np.zeros(0, np.uint32), np.zeros(nl, np.uint64), np.zeros(nl, np.uint64))
    p = str(tmp_path / "empty.v3")
    svdag_lib.items_to_v3(empty, p, svdag_lib.V3_CPU)
    with ref_mod.RefV3Dag(p) as r:
        assert r.root == 0xFFFFFFFF
        w, lw, li, found = r.items()
        assert int(li.sum()) == 0
