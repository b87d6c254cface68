"""The claim behind incremental served frames, checked with the oracle alone: after any edits, every
pixel whose primary ray meets none of the edits' boxes (as the server computes them: the footprint
grown by two voxels) keeps exactly its previous hit record. Cameras include axis-aligned views, whose
rays have zero direction components: those rays are always traced again (their intersection tests
compute NaN on node planes through the origin and can reach voxels off the ray), as the tracer does."""
import numpy as np
import pytest

LEVELS = 9
SCENE = dict(seed=2, octaves=5, num_materials=8, min_height_pct=35, max_height_pct=65)  # structures are 16-512 voxels:
# on a 512^3 grid one can swallow the camera


def boxes_of(e):
    """The server's edit_boxes, restated: [min xyz, max xyz] per changed region."""
    f = np.float32
    r = max(f(e.radius), f(0.1))
    lo, hi = r + f(2.0), r + f(3.0)
    c = np.array(list(e.center), dtype=np.float32)
    src, dst = np.array(list(e.src), dtype=np.float32), np.array(list(e.dst), dtype=np.float32)
    d = dst + (c - src)
    box = lambda p: np.concatenate([p - lo, p + hi]).astype(np.float32)
    if e.tool == 5:  # copy
        return [box(d)]
    if e.tool == 7:  # move
        return [box(c), box(d)]
    return [box(c)]


def rays(p):
    """Float rays of every pixel (x, y), as the tracer builds them."""
    W, H = p.width, p.height
    y, x = np.mgrid[0:H, 0:W].astype(np.float64)
    v = [((p.ray_min[i] + x * p.ray_ddx[i]) + y * p.ray_ddy[i]) - p.camera[i] for i in range(3)]
    inv = 1 / np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    with np.errstate(divide="ignore"):
        d = [(inv * v[i]).astype(np.float32) for i in range(3)]
        ivd = [np.float32(1.0) / d[i] for i in range(3)]
    o = [np.float32(p.camera[i]) for i in range(3)]
    return o, ivd


def meets(o, ivd, b):
    """ray_meets_box in float32 (fminf/fmaxf drop NaN like the device's)."""
    with np.errstate(invalid="ignore"):
        t1 = [(b[i] - o[i]) * ivd[i] for i in range(3)]
        t2 = [(b[3 + i] - o[i]) * ivd[i] for i in range(3)]
    tn = np.fmax(np.fmax(np.fmin(t1[0], t2[0]), np.fmin(t1[1], t2[1])), np.fmax(np.fmin(t1[2], t2[2]), np.float32(0)))
    tf = np.fmin(np.fmin(np.fmax(t1[0], t2[0]), np.fmax(t1[1], t2[1])), np.fmax(t1[2], t2[2]))
    return tn <= tf


def random_edit(oracle_mod, rng, L):
    g = 1 << LEVELS
    x, z = (int(v) for v in rng.integers(g // 4, 3 * g // 4, 2))  # where the cameras look
    h = L.oracle_terrain_height(oracle_mod.TerrainParams(**SCENE), LEVELS, x, z)
    e = oracle_mod.Edit()
    e.tool = int(rng.choice([0, 1, 2, 3, 4, 5, 7, 8]))
    e.material = int(rng.integers(0, 16))
    e.radius = float(rng.integers(2, 40))
    e.center[:] = [float(x), float(h + rng.integers(-6, 7)), float(z)]
    if e.tool in (5, 7):
        e.radius = min(e.radius, 16.0)
        e.src[:] = list(e.center)
        e.dst[:] = [e.center[0] + float(rng.integers(-40, 41)), e.center[1], e.center[2] + float(rng.integers(-40, 41))]
    if e.tool == 8:
        e.noise_seed = int(rng.integers(4, 20))
    return e


def camera(view, g):
    if view == "oblique":
        return (0.1 * g, 0.9 * g, 0.1 * g), (0.5 * g, 0.45 * g, 0.5 * g)
    if view == "down":
        return (0.5 * g, 1.2 * g, 0.5 * g), (0.5 * g, 0.0, 0.5 * g)
    if view == "side":
        return (0.5 * g, 0.8 * g, 0.05 * g), (0.5 * g, 0.4 * g, 0.5 * g)
    r = np.random.default_rng(int(view[-1]))  # "randomN": a seeded camera above the terrain
    eye = (float(r.uniform(0, g)), float(r.uniform(0.75, 1.2) * g), float(r.uniform(0, g)))
    return eye, (float(r.uniform(0.3, 0.7) * g), float(r.uniform(0.3, 0.5) * g), float(r.uniform(0.3, 0.7) * g))


@pytest.mark.parametrize("view", ["oblique", "down", "side", "random1", "random2", "random3", "random4"])
def test_untouched_pixels_keep_their_hits(oracle_mod, view):
    L = oracle_mod.lib()
    o = oracle_mod.OracleDag(LEVELS)
    o.build_terrain(oracle_mod.TerrainParams(**SCENE))
    g = float(1 << LEVELS)
    eye, target = camera(view, g)
    p = oracle_mod.camera_params(eye, target, 60.0, 96, 72)
    o_, ivd = rays(p)
    rng = np.random.default_rng(sum(map(ord, view)))
    prev = o.trace(p, threads=8)
    checked = changed = 0
    for wave in range(12):
        touched = ~((np.abs(ivd[0]) <= 1e30) & (np.abs(ivd[1]) <= 1e30) & (np.abs(ivd[2]) <= 1e30))
        for _ in range(int(rng.integers(1, 4))):
            e = random_edit(oracle_mod, rng, L)
            assert o.edit(e).status == 0
            for b in boxes_of(e):
                touched |= meets(o_, ivd, b)
        cur = o.trace(p, threads=8)
        keep = ~touched[::-1].reshape(-1)  # buffer row H - 1 - y holds pixel row y
        assert prev[keep].tobytes() == cur[keep].tobytes(), (view, wave)
        checked += int(keep.sum())
        changed += int((prev.view(np.uint8).reshape(len(prev), -1) != cur.view(np.uint8).reshape(len(cur), -1)).any(1).sum())
        prev = cur
    assert checked > 0 and changed > 100  # the edits do show in the frames
