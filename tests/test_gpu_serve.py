"""Serving form: every edit's result is the same alone and in the mix.

A request stream (add / remove / paint / copy, uneven radii) is served with continuous batching; the
root after each edit, read from the request results, must equal canonically the state the same
edits give one at a time through the plain per-edit path and through the oracle. The plain server
mode (one request per launch) must give the same states too.
"""
import numpy as np
import pytest

from gpu_util import gpu_canon, gpu_subtree_canon

pytestmark = pytest.mark.gpu

LEVELS = 11
SCENE = dict(seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70, num_structures=24,
             structure_seed=5)


def stream(n_rate, duration):
    import svdag.workloads as w

    return w.c4_stream(n_rate, duration, seed=12, levels=LEVELS, terrain=SCENE, rmax=96.0, copy_offset=64)


def to_oracle(oracle_mod, e):
    o = oracle_mod.Edit()
    o.tool, o.material, o.radius = e.tool, e.material, e.radius
    o.center[:], o.src[:], o.dst[:] = list(e.center), list(e.src), list(e.dst)
    o.noise_seed, o.noise_cell_log2 = e.noise_seed, e.noise_cell_log2
    return o


def states_alone(svdag_lib, oracle_mod, edits):
    g = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=2 << 30)
    g.build_terrain(**SCENE)
    o = oracle_mod.OracleDag(LEVELS)
    o.build_terrain(oracle_mod.TerrainParams(**SCENE))
    out = []
    for e in edits:
        g.edit(e)
        o.edit(to_oracle(oracle_mod, e))
        c = gpu_canon(oracle_mod, g)
        assert c == o.canon()
        out.append(c)
    g.free()
    return out


def served_states(svdag_lib, oracle_mod, edits, times, frames, plain):
    g = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=2 << 30, undo_depth=32)
    g.build_terrain(**SCENE)
    cam = svdag_lib.get_trace_params((1024.0, 1900.0, 300.0), (1024.0, 1100.0, 1024.0), 320, 180)
    with svdag_lib.Server(g, cam, max_batch=16, plain=plain) as srv:
        res = srv.replay(edits, times, frames)
    n = len(edits)
    assert (res["status"] == 0).all()
    assert (res["visible_s"] >= res["submit_s"]).all()
    states = [gpu_subtree_canon(oracle_mod, g, 0, int(r)) for r in res["root_after"][:n]]
    assert g.get_first_node_index() == int(res["root_after"][n - 1])
    launches = len(set(res["launch"][:n].tolist()))
    g.free()
    return states, launches


@pytest.mark.parametrize("burst", [False, True])
def test_served_edits_equal_alone(svdag_lib, oracle_mod, burst):
    times, edits, frames = stream(3000.0, 0.012)
    assert len(edits) >= 20
    if burst:  # everything arrives at once: the batches are as large as the slots allow
        times = [0.0] * len(edits)
    alone = states_alone(svdag_lib, oracle_mod, edits)
    served, launches = served_states(svdag_lib, oracle_mod, edits, times, frames, plain=False)
    assert served == alone
    if burst:
        assert launches < len(edits)
    plain, launches = served_states(svdag_lib, oracle_mod, edits, times, frames, plain=True)
    assert plain == alone
    assert launches == len(edits)
