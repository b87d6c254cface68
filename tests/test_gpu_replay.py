"""A recorded edit session (the reference's replay format, replay.h) served as requests.

The session is written in the reference's file format (camera moves, tool parameters, sphere / cube
/ paint / copy edits with and without their optional cells, undo, redo, fills, one EndFrame per
frame) on a replay grid one level coarser than the scene, parsed by the library and served with
continuous batching and by the plain one-request-at-a-time loop. Every edit, undo and redo must leave
the state the oracle reaches applying the same actions in order (MyGPUHashDAGUndoRedo semantics
included), and the last served frame must equal the oracle's trace of the final state.
"""
import numpy as np
import pytest

from gpu_util import compare_hits, gpu_subtree_canon

pytestmark = pytest.mark.gpu

LEVELS = 11
REPLAY_LEVELS = 10
SCENE = dict(seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70, num_structures=24,
             structure_seed=5)
BOUNDS = ((-1.0, -1.0, -1.0), (1.0, 1.0, 1.0))


def look_rows(pos, target):
    f = np.asarray(target, float) - np.asarray(pos, float)
    f /= np.linalg.norm(f)
    r = np.cross(f, [0.0, 1.0, 0.0])
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    return [float(v) for v in np.concatenate([-r, u, f])]


def session_csv(svdag_lib, frames, seed):
    """A session near the terrain surface, in replay-grid voxels (scene voxels / 2)."""
    rng = np.random.default_rng(seed)
    g = 1 << REPLAY_LEVELS
    lines = []
    f = lambda v: "%f" % v
    for _ in range(frames):
        if rng.random() < 0.3:
            pos = [float(v) for v in rng.uniform(-0.6, 0.6, 3)]
            pos[1] = float(rng.uniform(0.6, 0.9))
            lines.append("SetLocation," + ",".join(map(f, pos)))
            lines.append("SetRotation," + ",".join(map(f, look_rows(pos, (0.0, 0.1, 0.0)))))
        for _ in range(int(rng.integers(1, 4))):
            x, z = (int(v) for v in rng.integers(0, g, 2))
            y = svdag_lib.scene_height(LEVELS, 2 * x, 2 * z, **SCENE) / 2.0 + float(rng.integers(-8, 9))
            loc = [float(x), y, float(z)]
            r = float(rng.uniform(2.0, 24.0))
            u = rng.random()
            if u < 0.35:
                cells = loc + [r]
                cell = ",".join(map(f, cells)) + "," + ("true" if rng.random() < 0.5 else "false")
                if rng.random() < 0.7:
                    cell += ",%d" % int(rng.integers(0, 16))
                lines.append(("EditSphere," if rng.random() < 0.6 else "EditCube,") + cell)
            elif u < 0.55:
                cell = ",".join(map(f, loc + [r]))
                if rng.random() < 0.7:
                    cell += "," + ",".join(map(f, rng.uniform(0, 1, 3))) + ",%d" % int(rng.integers(0, 16))
                lines.append("EditPaint," + cell)
            elif u < 0.75:
                off = rng.integers(-48, 49, 2)
                dst = [loc[0] + float(off[0]), loc[1], loc[2] + float(off[1])]
                cell = ",".join(map(f, loc + loc + dst + [min(r, 16.0)]))
                if rng.random() < 0.5:
                    cell += ",1,0,0,0,1,0,0,0,1,false,1.000000"
                lines.append("EditCopy," + cell)
            elif u < 0.87:
                lines.append("Undo" if rng.random() < 0.6 else "Redo")
            elif u < 0.94:
                lines.append("SetToolParameters," + ",".join(str(int(v)) for v in rng.integers(0, g, 9)) + ",0," + f(r))
            else:
                lines.append("EditFill," + ",".join(map(f, loc + [r])))
        lines.append("EndFrame")
    return "\n".join(lines) + "\n"


def to_oracle(oracle_mod, e):
    o = oracle_mod.Edit()
    o.tool, o.material, o.radius = e.tool, e.material, e.radius
    o.center[:], o.src[:], o.dst[:] = list(e.center), list(e.src), list(e.dst)
    return o


def oracle_params(oracle_mod, p):
    po = oracle_mod.TraceParams()
    for name in ("camera", "ray_min", "ray_ddx", "ray_ddy"):
        getattr(po, name)[:] = list(getattr(p, name))
    po.width, po.height = p.width, p.height
    return po


@pytest.fixture(scope="module")
def session(svdag_lib, oracle_mod):
    acts = svdag_lib.parse_replay(session_csv(svdag_lib, 40, 21), svdag_lib.replay_scale(LEVELS, REPLAY_LEVELS))
    kinds = [a.kind for a in acts]
    assert kinds.count(svdag_lib.REPLAY_UNDO) >= 3 and kinds.count(svdag_lib.REPLAY_REDO) >= 2
    frames = svdag_lib.replay_frames(acts, 96, 64, LEVELS, *BOUNDS)
    o = oracle_mod.OracleDag(LEVELS)
    o.build_terrain(oracle_mod.TerrainParams(**SCENE))
    states = {}
    for i, a in enumerate(acts):
        if a.kind == svdag_lib.REPLAY_EDIT:
            assert o.edit(to_oracle(oracle_mod, a.edit)).status == 0
        elif a.kind == svdag_lib.REPLAY_UNDO:
            o.undo()
        elif a.kind == svdag_lib.REPLAY_REDO:
            o.redo()
        else:
            continue
        states[i] = o.canon()
    final_frame = o.trace(oracle_params(oracle_mod, frames[-1]), threads=8)
    return acts, frames, states, final_frame


@pytest.mark.parametrize("plain", [False, True])
def test_replayed_session_equals_oracle(svdag_lib, oracle_mod, session, plain):
    acts, frames, states, final_frame = session
    g = svdag_lib.MyGPUHashDAG(LEVELS, pool_bytes=2 << 30, undo_depth=32)
    g.build_terrain(**SCENE)
    with svdag_lib.Server(g, frames[0], max_batch=16, plain=plain, copy_frames=True) as srv:
        res = srv.replay_actions(acts, 0.0, frames)
        last = srv.frame()
    kinds = np.array([a.kind for a in acts])
    requests = np.isin(kinds, [svdag_lib.REPLAY_EDIT, svdag_lib.REPLAY_UNDO, svdag_lib.REPLAY_REDO,
                               svdag_lib.REPLAY_END_FRAME])
    assert (res["ticket"][requests] > 0).all() and (res["ticket"][~requests] == 0).all()
    want_kind = {svdag_lib.REPLAY_EDIT: 0, svdag_lib.REPLAY_END_FRAME: 1, svdag_lib.REPLAY_UNDO: 2,
                 svdag_lib.REPLAY_REDO: 3}
    for i in np.nonzero(requests)[0]:
        assert res["kind"][i] == want_kind[int(kinds[i])], i
    assert (res["status"][requests] == 0).all()
    for i, want in states.items():
        assert gpu_subtree_canon(oracle_mod, g, 0, int(res["root_after"][i])) == want, i
    last_state = max(states)
    assert g.get_first_node_index() == int(res["root_after"][last_state])
    launches = res["launch"][kinds == svdag_lib.REPLAY_EDIT]
    if plain:
        assert len(set(launches.tolist())) == len(launches)
    compare_hits(last, final_frame)
    g.free()
