"""Served frames traced only where the scene changed equal whole frames.

The server traces a frame of an unchanged camera only for pixels whose ray meets the bounding box of
an edit made since the previous frame. After every wave of edits (every tool, edits at the grid's
edges, a wave with no edit, an undo and a redo) the served frame must equal the oracle's trace of the
same state pixel by pixel (hit voxel and material exactly, positions within 1e-5 relative).
"""
import numpy as np
import pytest

from gpu_util import compare_hits

pytestmark = pytest.mark.gpu

LEVELS = 11
SCENE = dict(seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70, num_structures=24,
             structure_seed=5)


def to_oracle(oracle_mod, e):
    o = oracle_mod.Edit()
    o.tool, o.material, o.radius = e.tool, e.material, e.radius
    o.center[:], o.src[:], o.dst[:] = list(e.center), list(e.src), list(e.dst)
    o.noise_seed, o.noise_cell_log2 = e.noise_seed, e.noise_cell_log2
    return o


def oracle_params(oracle_mod, p):
    po = oracle_mod.TraceParams()
    for f in ("camera", "ray_min", "ray_ddx", "ray_ddy"):
        getattr(po, f)[:] = list(getattr(p, f))
    po.width, po.height = p.width, p.height
    return po


def waves(svdag_lib, rng):
    import svdag.workloads as w

    g = 1 << LEVELS
    tools = [svdag_lib.TOOL_SPHERE_ADD, svdag_lib.TOOL_SPHERE_REMOVE, svdag_lib.TOOL_BOX_ADD, svdag_lib.TOOL_BOX_REMOVE,
             svdag_lib.TOOL_SPHERE_PAINT, svdag_lib.TOOL_COPY, svdag_lib.TOOL_MOVE, svdag_lib.TOOL_SPHERE_ERODE]
    out = []
    for k in range(14):
        if k == 5:
            out.append([])  # a frame with no edit since the last one
            continue
        if k in (8, 9):
            out.append(["undo" if k == 8 else "redo"])
            continue
        wave = []
        for _ in range(int(rng.integers(1, 6))):
            edge = rng.random() < 0.25
            x = int(rng.choice([0, g - 1])) if edge else int(rng.integers(0, g))
            z = int(rng.integers(0, g))
            h = float(svdag_lib.scene_height(LEVELS, x, z, **SCENE))
            c = (float(x), h + float(rng.integers(-8, 9)), float(z))
            tool = int(rng.choice(tools))
            r = float(rng.integers(2, 48))
            if tool in (svdag_lib.TOOL_COPY, svdag_lib.TOOL_MOVE):
                off = rng.integers(-96, 97, 2)
                dst = (c[0] + float(off[0]), c[1], c[2] + float(off[1]))
                e = w.make_edit(tool, 0, c, min(r, 24.0), src=c, dst=dst)
            elif tool == svdag_lib.TOOL_SPHERE_ERODE:
                e = w.make_edit(tool, 0, c, r, noise_seed=int(rng.integers(4, 20)))
            else:
                e = w.make_edit(tool, int(rng.integers(0, 16)), c, r)
            wave.append(e)
        out.append(wave)
    return out


def test_incremental_frames_equal_whole_frames(svdag_lib, oracle_mod):
    rng = np.random.default_rng(31)
    g = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=2 << 30, undo_depth=32)
    g.build_terrain(**SCENE)
    o = oracle_mod.OracleDag(LEVELS)
    o.build_terrain(oracle_mod.TerrainParams(**SCENE))
    cam = svdag_lib.get_trace_params((-200.0, 1700.0, -150.0), (1024.0, 1000.0, 1024.0), 256, 192)
    po = oracle_params(oracle_mod, cam)
    with svdag_lib.Server(g, cam, max_batch=4, copy_frames=True) as srv:
        t = srv.submit_frame()
        srv.poll(t)
        compare_hits(srv.frame(), o.trace(po, threads=8))
        for wave in waves(svdag_lib, rng):
            tickets = []
            for e in wave:
                if e in ("undo", "redo"):
                    tickets.append(srv.submit_undo(redo=e == "redo"))
                    (o.undo if e == "undo" else o.redo)()
                else:
                    tickets.append(srv.submit_edit(e))
                    assert o.edit(to_oracle(oracle_mod, e)).status == 0
            tickets.append(srv.submit_frame())
            for tk in tickets:
                assert srv.poll(tk).status == 0
            compare_hits(srv.frame(), o.trace(po, threads=8))
        c = srv.counters()
        # the first frame and the undo/redo waves are whole, the other waves incremental
        assert c["frames_whole"] >= 3 and c["frames_incremental"] >= 8
        whole_bytes = 256 * 192 * 68
        assert whole_bytes * c["frames_whole"] <= c["frame_bytes_to_host"] < whole_bytes * (c["frames_whole"] + c["frames_incremental"])
    g.free()
