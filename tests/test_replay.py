"""Replay files (the reference's recorded edit sessions, replay.h) parsed by the library's host parser.

The expected actions come from a plain-Python restatement of ReplayManager::load_csv
(replay.h:650-683) and of the loaders of each action (replay.h:180-560), applied to files written
the way ReplayManager::write_csv (replay.h:620-632) writes them (std::to_string of floats).
"""
import ctypes as C
import glob
import math
import os

import numpy as np
import pytest


def to_string(v):
    """std::to_string: floats as %f, ints and booleans as the reference writes them."""
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, float):
        return "%f" % v
    return str(v)


def write_csv(actions):
    return "".join(name + "".join("," + to_string(v) for v in data) + "\n" for name, data in actions)


def expected(name, cells, scale):
    """The request one line becomes: (kind, tool, material, centre, radius, src, dst) or camera."""
    f = [float(c) for c in cells[:10]] if name not in ("EditSphere", "EditCube") else None
    if name == "EndFrame":
        return ("end",)
    if name in ("Undo", "Redo"):
        return (name.lower(),)
    if name in ("SetLocation", "SetRotation"):
        return ("camera", tuple(np.float32(v) for v in f))
    if name in ("SetToolParameters", "EditFill"):
        return ("other",)
    s = np.float32(scale)
    if name in ("EditSphere", "EditCube"):
        loc = [np.float32(float(c)) for c in cells[:3]]
        add = cells[4] in ("true", "TRUE")
        mat = int(cells[5]) if len(cells) > 5 else 1
        tool = {("EditSphere", True): 0, ("EditSphere", False): 1, ("EditCube", True): 2, ("EditCube", False): 3}[name, add]
        return ("edit", tool, mat, tuple(v * s for v in loc), np.float32(float(cells[3])) * s, None, None)
    if name == "EditPaint":
        mat = int(cells[7]) if len(cells) > 7 else 1
        return ("edit", 4, mat, tuple(np.float32(v) * s for v in f[:3]), np.float32(f[3]) * s, None, None)
    assert name == "EditCopy"
    return ("edit", 5, 0, tuple(np.float32(v) * s for v in f[:3]), np.float32(f[9]) * s,
            tuple(np.float32(v) * s for v in f[3:6]), tuple(np.float32(v) * s for v in f[6:9]))


def load_csv(text, scale):
    """ReplayManager::load_csv: split on ',' up to each '\\n', drop trailing empty cells."""
    out, data = [], []
    for c in text:
        if c == "\n":
            name, cells = data[0], data[1:]
            while cells and cells[-1] == "":
                cells.pop()
            out.append(expected(name, cells, scale))
            data = []
        elif c == ",":
            data.append("")
        else:
            if not data:
                data.append("")
            data[-1] += c
    return out


def as_tuple(a):
    import svdag

    if a.kind == svdag.REPLAY_END_FRAME:
        return ("end",)
    if a.kind == svdag.REPLAY_UNDO:
        return ("undo",)
    if a.kind == svdag.REPLAY_REDO:
        return ("redo",)
    if a.kind == svdag.REPLAY_CAMERA_LOCATION:
        return ("camera", tuple(np.float32(v) for v in a.camera[:3]))
    if a.kind == svdag.REPLAY_CAMERA_ROTATION:
        return ("camera", tuple(np.float32(v) for v in a.camera[:9]))
    if a.kind == svdag.REPLAY_OTHER:
        return ("other",)
    e = a.edit
    copy = e.tool == svdag.TOOL_COPY
    return ("edit", e.tool, e.material, tuple(np.float32(v) for v in e.center), np.float32(e.radius),
            tuple(np.float32(v) for v in e.src) if copy else None, tuple(np.float32(v) for v in e.dst) if copy else None)


def random_session(rng, frames, extent):
    """A recorded session: camera moves, tool parameters, every edit kind with and without its
    optional cells, undo/redo and fills, one EndFrame per frame."""
    acts = []
    for _ in range(frames):
        if rng.random() < 0.5:
            acts.append(("SetLocation", [float(v) for v in rng.uniform(-1, 1, 3)]))
            acts.append(("SetRotation", [float(v) for v in rng.uniform(-1, 1, 9)]))
        for _ in range(int(rng.integers(0, 4))):
            loc = [float(v) for v in rng.uniform(0, extent, 3)]
            r = float(rng.uniform(1, 32))
            u = rng.random()
            if u < 0.3:
                data = loc + [r, bool(rng.integers(0, 2))]
                if rng.random() < 0.5:
                    data.append(int(rng.integers(0, 16)))
                acts.append(("EditSphere" if rng.random() < 0.6 else "EditCube", data))
            elif u < 0.5:
                data = loc + [r]
                k = rng.random()
                if k < 0.3:
                    data += [float(v) for v in rng.uniform(0, 1, 3)]
                elif k < 0.6:
                    data += [float(v) for v in rng.uniform(0, 1, 3)] + [int(rng.integers(0, 16))]
                acts.append(("EditPaint", data))
            elif u < 0.7:
                data = loc + [float(v) for v in rng.uniform(0, extent, 6)] + [r]
                if rng.random() < 0.5:  # transform, swirl, period (ignored by the GPU copy editor)
                    data += [float(v) for v in rng.uniform(-1, 1, 9)] + [bool(rng.integers(0, 2)), float(r)]
                acts.append(("EditCopy", data))
            elif u < 0.8:
                acts.append(("Undo" if rng.random() < 0.5 else "Redo", []))
            elif u < 0.9:
                acts.append(("SetToolParameters", [float(v) for v in rng.uniform(0, 8, 11)]))
            else:
                acts.append(("EditFill", [float(v) for v in rng.uniform(0, extent, 3)] + [r]))
        acts.append(("EndFrame", []))
    return acts


def test_parse_matches_load_csv_restatement(svdag_lib):
    rng = np.random.default_rng(12)
    acts = random_session(rng, 200, 512.0)
    text = write_csv(acts)
    for scale in (1.0, svdag_lib.replay_scale(17, 13)):
        got = [as_tuple(a) for a in svdag_lib.parse_replay(text, scale)]
        assert got == load_csv(text, scale)
    assert svdag_lib.replay_scale(17, 13) == 16.0


def test_defaults_trailing_cells_and_line_endings(svdag_lib):
    s = svdag_lib
    text = ("EditSphere,1.5,2,3,4,true\nEditCube,1,2,3,4,FALSE,,,\r\n\nEditPaint,1,2,3,4,0.5,0.5,0.5\n"
            "Undo,\nRedo\nEndFrame,,\nEditPaint,1,2,3,4,0.5,0.5,0.5,7\nEndFrame")
    acts = s.parse_replay(text, 2.0)  # the unterminated last line is not an action (load_csv)
    assert [a.kind for a in acts] == [s.REPLAY_EDIT, s.REPLAY_EDIT, s.REPLAY_EDIT, s.REPLAY_UNDO, s.REPLAY_REDO,
                                      s.REPLAY_END_FRAME, s.REPLAY_EDIT]
    assert acts[0].edit.tool == s.TOOL_SPHERE_ADD and acts[0].edit.material == 1
    assert list(acts[0].edit.center) == [3.0, 4.0, 6.0] and acts[0].edit.radius == 8.0
    assert acts[1].edit.tool == s.TOOL_BOX_REMOVE
    assert acts[2].edit.tool == s.TOOL_SPHERE_PAINT and acts[2].edit.material == 1
    assert acts[6].edit.material == 7


@pytest.mark.parametrize("line", ["Jump,1,2", "EditSphere,1,2,3,4", "EditSphere,1,2,3,4,yes", "EditSphere,1,2,3,4,true,16",
                                  "EditCopy,1,2,3,4,5,6,7,8,9", "EditPaint,1,2,3,4,5", "SetLocation,1,2",
                                  "SetRotation,1,2,3,4,5,6,7,8", "EditSphere,a,2,3,4,true", "SetToolParameters,1,2",
                                  "EditCopy,1,2,3,4,5,6,7,8,9,10,1,0,0,0,1,0,0,0,1,maybe,1", "EditFill,1,2,x,4"])
def test_rejected_lines_name_their_line(svdag_lib, line):
    L = svdag_lib.lib()
    text = ("EndFrame\nUndo\n" + line + "\nEndFrame\n").encode()
    count, bad = C.c_uint64(), C.c_uint64()
    assert L.svdag_replay_parse(text, len(text), 1.0, None, 0, C.byref(count), C.byref(bad)) == 1
    assert bad.value == 2 and count.value == 2


def test_capacity_and_arguments(svdag_lib):
    L = svdag_lib.lib()
    text = b"Undo\nRedo\nEndFrame\n"
    out = (svdag_lib.ReplayAction * 2)()
    count = C.c_uint64()
    assert L.svdag_replay_parse(text, len(text), 1.0, C.addressof(out), 2, C.byref(count), None) == 2  # OOM
    assert count.value == 3 and out[1].kind == svdag_lib.REPLAY_REDO
    assert L.svdag_replay_parse(text, len(text), 0.0, None, 0, C.byref(count), None) == 1
    assert L.svdag_replay_parse(text, len(text), 1.0, None, 0, None, None) == 1
    assert L.svdag_replay_parse(None, 0, 1.0, None, 0, C.byref(count), None) == 0 and count.value == 0


def test_view_trace_params_equal_look_at(svdag_lib):
    """CameraView rows (right = -row 0, up = row 1, forward = row 2) give the look-at basis."""
    pos = np.array([0.1, 0.3, -0.2])
    fwd = np.array([0.3, -0.2, 0.9])
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, [0.0, 1.0, 0.0])
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    rot = np.concatenate([-right, up, fwd]).astype(np.float32)
    pos = pos.astype(np.float32)
    a = svdag_lib.view_trace_params(pos, rot, 64, 48, 10, (-1, -1, -1), (1, 1, 1))
    b = svdag_lib.get_trace_params(pos.astype(np.float64), pos.astype(np.float64) + rot[6:9].astype(np.float64), 64, 48,
                                   levels=10, bounds_min=(-1, -1, -1), bounds_max=(1, 1, 1))
    for f in ("camera", "ray_min", "ray_ddx", "ray_ddy"):
        assert np.allclose(list(getattr(a, f)), list(getattr(b, f)), rtol=1e-5, atol=1e-5), f
    frames = svdag_lib.replay_frames(svdag_lib.parse_replay("EndFrame\nSetLocation,1,2,3\nEndFrame\n"), 8, 8, 4,
                                     (0, 0, 0), (16, 16, 16))
    assert len(frames) == 2 and list(frames[1].camera) == [1.0, 2.0, 3.0]


def _replays_dir():
    """The reference's replays/ folder: SVDAG_REFERENCE_REPLAYS, else beside the reference sources
    the oracle/_ref recipe compiles (absent on machines without the reference)."""
    if os.environ.get("SVDAG_REFERENCE_REPLAYS"):
        return os.environ["SVDAG_REFERENCE_REPLAYS"]
    import importlib.util

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("build_ref", os.path.join(root, "oracle", "build_ref.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return os.path.join(os.path.dirname(mod.REFERENCE_SRC), "replays")


REPLAYS = _replays_dir()


@pytest.mark.skipif(not os.path.isdir(REPLAYS), reason="the reference's replay files are not on this machine")
def test_reference_replays_parse_like_load_csv(svdag_lib):
    """Every recorded session of the reference parses, with the same actions as the restatement
    (sessions whose materials exceed the GPU path's 16 are reported as rejected)."""
    files = sorted(glob.glob(os.path.join(REPLAYS, "*.csv")))
    assert files
    parsed = 0
    for path in files:
        text = open(path, newline="").read()
        try:
            want = load_csv(text, 1.0)
        except (ValueError, KeyError, IndexError):
            continue
        if any(w[0] == "edit" and not (0 <= w[2] < 16) for w in want):
            with pytest.raises(svdag_lib.SvdagError):
                svdag_lib.parse_replay(text, 1.0)
            continue
        got = [as_tuple(a) for a in svdag_lib.parse_replay(text, 1.0)]
        assert got == want, path
        parsed += 1
    assert parsed > 0
    assert not math.isnan(parsed)
