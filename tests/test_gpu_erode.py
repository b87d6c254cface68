"""The erosion tool (MyGpuSphereErosionEditor, my_gpu_dag_editors.h:538-589) against the oracle: the
DAG after every edit canonically, the per-edit counters exactly, voxels in bricks around the sphere.
Neighbour counts read the DAG before the edit, and coordinates off the grid wrap around it (the
reference's unsigned paths), which the edit at the grid corner exercises."""
import numpy as np
import pytest

from gpu_util import gpu_canon, gpu_sample

pytestmark = pytest.mark.gpu

LEVELS = 10
SCENE = dict(seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70, num_structures=32,
             structure_seed=9)


def erode(svdag_lib, center, radius, threshold):
    return svdag_lib.MyGpuSphereErosionEditor(center, radius, threshold).to_edit()


def to_oracle(oracle_mod, e):
    o = oracle_mod.Edit()
    o.tool, o.material, o.radius, o.noise_seed = e.tool, e.material, e.radius, e.noise_seed
    o.center[:] = list(e.center)
    return o


def edits(svdag_lib):
    h = lambda x, z: float(svdag_lib.scene_height(LEVELS, x, z, **SCENE))
    return [
        erode(svdag_lib, (300.0, h(300, 300), 300.0), 20.0, 13),
        erode(svdag_lib, (640.0, h(640, 200), 200.0), 36.0, 6),
        erode(svdag_lib, (100.0, h(100, 800) - 10.0, 800.0), 14.0, 20),
        erode(svdag_lib, (0.0, 2.0, 0.0), 9.0, 10),  # the grid corner: neighbours wrap around
        erode(svdag_lib, (512.0, h(512, 512), 512.0), 28.0, 25),
    ]


@pytest.mark.parametrize("form", ["graph", "persistent", "batch"])
def test_erosion_matches_oracle(svdag_lib, oracle_mod, form):
    g = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=2 << 30, persistent=form == "persistent")
    g.build_terrain(**SCENE)
    o = oracle_mod.OracleDag(LEVELS)
    o.build_terrain(oracle_mod.TerrainParams(**SCENE))
    es = edits(svdag_lib)
    if form == "batch":
        for e in es:
            o.edit(to_oracle(oracle_mod, e))
        g.edit_batch(es)
        assert gpu_canon(oracle_mod, g) == o.canon()
    else:
        for e in es:
            so = o.edit(to_oracle(oracle_mod, e))
            g.edit(e)
            sg = g.last_edit_stats()
            assert sg.status == 0
            assert list(sg.svo_nodes) == list(so.svo_nodes)
            assert (sg.unique_items, sg.new_items, sg.edited_voxels) == (so.unique_items, so.new_items, so.edited_voxels)
            assert gpu_canon(oracle_mod, g) == o.canon()
    rng = np.random.default_rng(4)
    r = np.arange(-40, 41, 4)
    for e in es:
        c = np.array(list(e.center), dtype=np.int64)
        pts = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3) + c + rng.integers(0, 4, 3)
        xyz = (pts % (1 << LEVELS)).astype(np.uint32)
        assert np.array_equal(gpu_sample(g, xyz), o.sample(xyz))
    g.free()


def test_erosion_removes_exposed_voxels(svdag_lib):
    """With threshold 25 only voxels whose 26 neighbours are all filled stay inside the sphere; an
    isolated voxel goes with threshold 0; voxels outside the sphere are untouched."""
    g = svdag_lib.MyGPUHashDAG(8, pool_bytes=512 << 20)
    # [69, 189)^3: not aligned to leaves (a box of whole leaves builds no leaves and, as in the
    # reference, leaves the DAG unchanged)
    g.edit(svdag_lib.MyGpuBoxEditor((129.0, 129.0, 129.0), 60.0, 3, True).to_edit())
    g.edit(svdag_lib.MyGpuBoxEditor((30.0, 30.0, 30.0), 0.0, 5, True).to_edit())  # one voxel
    g.edit(svdag_lib.MyGpuSphereErosionEditor((129.0, 160.0, 129.0), 40.0, 25).to_edit())
    g.edit(svdag_lib.MyGpuSphereErosionEditor((30.0, 30.0, 30.0), 5.0, 0).to_edit())
    xyz = np.array([[129, 160, 129], [129, 188, 129], [71, 188, 71], [30, 30, 30]], dtype=np.uint32)
    got = gpu_sample(g, xyz)
    assert got[0] == 3  # inside the box and the sphere, all neighbours filled
    assert got[1] == 0xFFFFFFFF  # the box's top face inside the sphere: exposed, removed
    assert got[2] == 3  # the top face outside the sphere
    assert got[3] == 0xFFFFFFFF  # the isolated voxel
    g.free()
