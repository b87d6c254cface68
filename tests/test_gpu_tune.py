"""Autotuner of the batched form: it picks a supported setting, gives back the space of its scratch
tables, and the edits it times are applied exactly as the plain path applies them."""
import numpy as np
import pytest

from gpu_util import TERRAIN, gpu_canon

pytestmark = pytest.mark.gpu


def node_keys(rng, n):
    keys = []
    for p in rng.integers(1, 9, n):
        bits = rng.choice(8, size=p, replace=False)
        keys.append((int(sum(1 << int(b) for b in bits)),) + tuple(int(v) for v in rng.integers(0, 1 << 28, p)))
    return keys


def test_table_tuning_picks_a_setting_and_returns_its_space(svdag_lib):
    import torch

    g = svdag_lib.MyGPUHashDAG(10, pool_bytes=1 << 30)
    g.build_terrain(**TERRAIN)
    used = g.stats().item_region_used_bytes
    rng = np.random.default_rng(8)
    keys = node_keys(rng, 200000)
    words = np.concatenate([np.array(k, dtype=np.uint32) for k in keys])
    offs = np.cumsum([0] + [len(k) for k in keys[:-1]]).astype(np.uint32)
    dw = torch.from_numpy(words.view(np.int32)).cuda()
    do = torch.from_numpy(offs.view(np.int32)).cuda()
    t = g.autotune(keys=dw, offsets=do, n_keys=len(keys), total_words=len(words), kind=svdag_lib.KIND_NODE)
    assert t.trials == 20
    assert t.load_factor in (8, 12, 16, 24, 32)
    assert t.probe_lanes in (1, 2, 4, 8)
    assert t.table_ns_per_key > 0
    assert g.stats().item_region_used_bytes == used
    cur = g.tuning()
    assert (cur.load_factor, cur.probe_lanes) == (t.load_factor, t.probe_lanes)
    # a table created afterwards still works with the tuned lanes
    tbl = g.create_table(svdag_lib.KIND_NODE, [64] * 9)
    out = torch.empty(len(keys), dtype=torch.int32, device="cuda")
    tbl.add(dw, do, len(keys), len(words), out)
    tbl.find(dw, do, len(keys), len(words), out)
    torch.cuda.synchronize()
    assert (out.cpu().numpy().view(np.uint32) != 0xFFFFFFFF).all()
    g.free()


def test_edit_tuning_applies_the_sample_like_the_plain_path(svdag_lib, oracle_mod):
    import svdag.workloads as w

    edits = [w.make_edit(tool, mat, c, r) for tool, mat, c, r in w.c0_edits(24)]
    g = svdag_lib.MyGPUHashDAG(10, pool_bytes=1 << 30)
    g.build_terrain(**TERRAIN)
    t = g.autotune(edits=edits)
    assert t.trials == len(edits)
    assert t.graph_us_small > 0 and t.persistent_us_small > 0
    assert t.persistent_leaves in (0, 1024, 4096, 16384, 65536)
    o = oracle_mod.OracleDag(10)
    o.build_terrain(oracle_mod.TerrainParams(**TERRAIN))
    for e in edits:
        oe = oracle_mod.Edit(tool=e.tool, material=e.material, radius=e.radius)
        oe.center[:] = list(e.center)
        o.edit(oe)
    assert gpu_canon(oracle_mod, g) == o.canon()
    assert g.stats().undo_count == o.undo_count()  # frames pushed as the plain path pushes them
    g.free()
