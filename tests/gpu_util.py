"""Shared helpers of the GPU parity tests (test infrastructure)."""
import numpy as np

TERRAIN = dict(seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70)


def gpu_canon(oracle_mod, dag):
    levels = dag.levels
    dumps = [dag.export_level(l) for l in range(levels - 1)]
    root = dag.get_first_node_index()
    if root == 0xFFFFFFFF:
        return oracle_mod.Canon().as_dict(levels)
    return oracle_mod.canonicalize_dump(levels, root, dumps)


def gpu_read(dag, level, handles):
    """Item words (n, 10) of the given handles of one level."""
    import torch

    h = torch.from_numpy(np.ascontiguousarray(handles, dtype=np.uint32).view(np.int32)).cuda()
    out = torch.empty((len(handles), 10), dtype=torch.int32, device="cuda")
    dag.table(level).read(h, len(handles), out)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32)


def gpu_node_at(dag, level, path):
    """Handle of the node (level, path) of the GPU DAG, or None where the subtree is empty."""
    h = dag.get_first_node_index()
    for l in range(level):
        if h == 0xFFFFFFFF:
            return None
        w = gpu_read(dag, l, [h])[0]
        s = level - l - 1
        c = (((path[0] >> s) & 1) << 2) | (((path[1] >> s) & 1) << 1) | ((path[2] >> s) & 1)
        mask = int(w[0]) & 0xFF
        if not (mask >> c) & 1:
            return None
        h = int(w[1 + bin(mask & ((1 << c) - 1)).count("1")])
    return h


def gpu_subtree_canon(oracle_mod, dag, level, handle):
    """Canonical form of the GPU DAG's subtree under `handle` (an item of `level`), read item by item."""
    levels = dag.levels
    empty = (np.zeros(0, np.uint32), np.zeros((0, 10), np.uint32))
    dumps = [empty] * (levels - 1)
    frontier = np.array([handle], dtype=np.uint32)
    for l in range(level, levels - 1):
        words = gpu_read(dag, l, frontier)
        dumps[l] = (frontier, words)
        if l == levels - 2:
            break
        pc = np.array([bin(int(m) & 0xFF).count("1") for m in words[:, 0]])
        kids = np.concatenate([words[i, 1:1 + pc[i]] for i in range(len(frontier))])
        frontier = np.unique(kids).astype(np.uint32)
    return oracle_mod.canonicalize_dump(levels, handle, dumps, level)


def random_bricks(rng, levels, n, size=16):
    g = 1 << levels
    lo = rng.integers(0, g - size, size=(n, 3))
    r = np.arange(size)
    x, y, z = np.meshgrid(r, r, r, indexing="ij")
    off = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    return (lo[:, None, :] + off[None, :, :]).reshape(-1, 3).astype(np.uint32)


def gpu_sample(dag, xyz):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(xyz, dtype=np.uint32).view(np.int32)).cuda()
    out = torch.empty(len(xyz), dtype=torch.int32, device="cuda")
    dag.sample_voxels(t, len(xyz), out)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32)


def gpu_trace(svdag, dag, params):
    tracer = svdag.DAGTracer(params.width, params.height)
    tracer.resolve_paths(params, dag)
    import torch

    torch.cuda.synchronize()
    return tracer.hits_numpy()


def sphere_edits(oracle_mod, levels, n, seed, terrain=TERRAIN, rmin=4, rmax=64, near=32):
    """C0 edit stream: centres within +-near voxels of the surface, integer radius U[rmin, rmax],
    50% add / 50% remove, add material U[0, 8)."""
    L = oracle_mod.lib()
    p = oracle_mod.TerrainParams(**terrain)
    rng = np.random.default_rng(seed)
    g = 1 << levels
    edits = []
    for _ in range(n):
        x, z = (int(v) for v in rng.integers(0, g, 2))
        h = L.oracle_terrain_height(p, levels, x, z)
        cx = x + int(rng.integers(-near, near + 1))
        cy = h + int(rng.integers(-near, near + 1))
        cz = z + int(rng.integers(-near, near + 1))
        r = int(rng.integers(rmin, rmax + 1))
        add = bool(rng.integers(0, 2))
        mat = int(rng.integers(0, 8))
        edits.append((0 if add else 1, mat, (float(cx), float(cy), float(cz)), float(r)))
    return edits


def to_oracle_edit(oracle_mod, tool, mat, center, radius, **kw):
    e = oracle_mod.Edit(tool=tool, material=mat)
    e.center[:] = list(center)
    e.radius = radius
    for k, v in kw.items():
        if k in ("src", "dst"):
            getattr(e, k)[:] = list(v)
        else:
            setattr(e, k, v)
    return e


def to_svdag_edit(svdag, tool, mat, center, radius, **kw):
    e = svdag.Edit(tool=tool, material=mat)
    e.center[:] = list(center)
    e.radius = radius
    for k, v in kw.items():
        if k in ("src", "dst"):
            getattr(e, k)[:] = list(v)
        else:
            setattr(e, k, v)
    return e


def compare_hits(a, b, rel=1e-5):
    """Exact voxel path and material on every pixel; hit position within `rel` relative (it is in
    fact bit-identical). Rays with a zero direction component produce NaN positions (0 * inf in the
    reference's createSurfaceInteraction, tracer.cu:353-389); NaN must appear at the same pixels."""
    assert np.array_equal(a["path"], b["path"])
    hit = np.any(a["path"] != 0, axis=1)
    assert np.array_equal(a["material"][hit], b["material"][hit])
    for f in ("position", "normal", "dpdu", "dpdv"):
        pa, pb = a[f].astype(np.float64), b[f].astype(np.float64)
        na, nb = np.isnan(pa), np.isnan(pb)
        assert np.array_equal(na, nb), f
        ok = ~na
        scale = np.maximum(np.abs(pa[ok]), 1.0)
        assert np.all(np.abs(pa[ok] - pb[ok]) <= rel * scale), f
