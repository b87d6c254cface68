"""The oracle pinned to the reference's own code (oracle/_ref, built from the reference sources by
oracle/build_ref.py).

Every function compared here runs reference code on the host: the editors' should_edit and
get_new_value (my_gpu_dag_editors.h), LeafBuilder_ and the header codecs (my_gpu_base_dag.h:86-351),
DAGUtils::get_value (dag_utils.h:146-182). The oracle must agree with it exactly:
  - every editor decision on a million seeded (tool, node, state) cases, a third of them placed on
    the sphere or box boundary where float rounding decides;
  - leaves and node headers built by LeafBuilder_ / encode_node_header, word for word;
  - voxel values of the oracle's DAG read through the reference's get_value;
  - after edits of every reference tool, the oracle's voxels equal what the reference editors decide
    voxel by voxel over the DAG before the edit (create_edit_svo.cu's per-node and per-voxel rules).
Skipped where the reference sources are absent and the harness was not built.
"""
import ctypes as C

import numpy as np
import pytest

from gpu_util import TERRAIN


@pytest.fixture(scope="module")
def ref_mod(oracle_mod):
    from oracle import ref

    if ref.lib() is None:
        pytest.skip("oracle/_ref is not built here (the reference sources are absent)")
    return ref


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def make_edit(oracle_mod, tool, material, center, radius, src=(0, 0, 0), dst=(0, 0, 0), threshold=0):
    e = oracle_mod.Edit(tool=tool, material=material, radius=float(radius), noise_seed=threshold)
    e.center[:] = [float(v) for v in center]
    e.src[:] = [float(v) for v in src]
    e.dst[:] = [float(v) for v in dst]
    return e


def decision_cases(rng, n, levels=17):
    """(edits, paths, depths, states, fills): per edit a batch of nodes; a third of the nodes sit on
    the editor's boundary (node corners at the sphere radius or on the box faces)."""
    tools = [0, 1, 2, 3, 4, 5, 8]
    g = 1 << levels
    out = []
    per = 2000
    for i in range(n // per):
        tool = tools[i % len(tools)]
        kind = rng.integers(0, 3)
        if kind == 0:  # integer centre and radius
            c = rng.integers(0, g, 3).astype(np.float32)
            r = float(rng.integers(0, 300))
        elif kind == 1:  # half-integer centre, fractional radius
            c = (rng.integers(0, g, 3) + 0.5).astype(np.float32)
            r = float(np.float32(rng.uniform(0.0, 300.0)))
        else:  # arbitrary floats
            c = rng.uniform(0, g, 3).astype(np.float32)
            r = float(np.float32(rng.uniform(0.0, 2000.0)))
        e_args = dict(tool=tool, material=int(rng.integers(0, 16)), center=c, radius=r,
                      src=rng.integers(0, g, 3), dst=rng.integers(0, g, 3), threshold=int(rng.integers(0, 27)))
        depth = rng.integers(0, 12, per).astype(np.uint32)
        # nodes around the centre: offsets of a few radii, some exactly at the radius along an axis
        off = rng.uniform(-2.5, 2.5, (per, 3)) * max(r, 1.0)
        edge = rng.random(per) < 0.33
        axis = rng.integers(0, 3, per)
        sgn = np.where(rng.random(per) < 0.5, -1.0, 1.0)
        off[edge] = 0.0
        off[edge, axis[edge]] = sgn[edge] * r
        pos = np.clip(c[None, :] + off, 0, g - 1).astype(np.int64)
        paths = (pos >> depth[:, None]).astype(np.uint32)
        states = rng.integers(0, 3, per).astype(np.uint32)
        fills = rng.integers(0, 16, per).astype(np.uint32)
        out.append((e_args, np.ascontiguousarray(paths), depth, states, fills))
    return out


def test_editor_decisions_equal_the_reference_editors(oracle_mod, ref_mod):
    rng = np.random.default_rng(20240611)
    L, R = oracle_mod.lib(), ref_mod.lib()
    total = 0
    for e_args, paths, depth, states, fills in decision_cases(rng, 1_000_000):
        e = make_edit(oracle_mod, **e_args)
        n = len(depth)
        o_ops, r_ops = np.empty(n, np.int32), np.empty(n, np.int32)
        o_f, r_f = np.empty(n, np.uint32), np.empty(n, np.uint32)
        L.oracle_should_edit_many(C.byref(e), _p(paths), _p(depth), _p(states), _p(fills), n, _p(o_ops), _p(o_f))
        assert R.ref_should_edit_many(C.byref(e), _p(paths), _p(depth), _p(states), _p(fills), n, _p(r_ops), _p(r_f)) == 0
        bad = np.nonzero(o_ops != r_ops)[0]
        assert len(bad) == 0, (e_args, paths[bad[0]], depth[bad[0]], states[bad[0]], o_ops[bad[0]], r_ops[bad[0]])
        fill = (o_ops == 1)
        assert np.array_equal(o_f[fill], r_f[fill]), e_args
        total += n
    assert total >= 1_000_000


def test_leaf_and_header_codecs_equal_the_reference(oracle_mod, ref_mod):
    rng = np.random.default_rng(7)
    L, R = oracle_mod.lib(), ref_mod.lib()
    for i in range(20000):
        p = [0.0, 0.02, 0.5, 0.98, 1.0][i % 5]
        filled = rng.random(64) < p
        mats = rng.integers(0, 16, 64).astype(np.uint32)
        ref_in = np.where(filled, mats, 0xFFFFFFFF).astype(np.uint32)
        ref_out = np.zeros(10, np.uint32)
        n_ref = R.ref_build_leaf(_p(ref_in), _p(ref_out))
        mask = int(sum(1 << v for v in range(64) if filled[v]))
        dense = np.ascontiguousarray(mats)
        or_out = np.zeros(10, np.uint32)
        n_or = L.oracle_build_leaf(mask, _p(dense), _p(or_out))
        assert n_ref == n_or and np.array_equal(ref_out[:n_ref], or_out[:n_or]), (i, mask)
        assert R.ref_leaf_size(_p(ref_out)) == L.oracle_leaf_size(_p(or_out)) == n_ref
        for v in range(0, 64, 7):
            a, b = C.c_uint32(), C.c_uint32()
            ra = R.ref_leaf_material(_p(ref_out), v, C.byref(a))
            ob = L.oracle_leaf_material(_p(or_out), v, C.byref(b))
            assert ra == ob and (not ra or a.value == b.value)
    for mask in range(256):
        for payload in (0, 1, 0x1234, (1 << 19) - 1):
            assert R.ref_encode_node_header(mask, payload) == L.oracle_encode_node_header(mask, payload)
        for m in range(16):
            h = R.ref_encode_full_node_header(mask, m)
            out = C.c_uint32()
            assert R.ref_header_fully_filled(h, C.byref(out)) == 1 and out.value == m
            assert h == (mask | (1 << 8) | (m << 9))  # the layout the oracle and the CUDA library write


def oracle_scene(oracle_mod, levels=10):
    o = oracle_mod.OracleDag(levels)
    o.build_terrain(oracle_mod.TerrainParams(**TERRAIN))
    return o


def surface_centre(oracle_mod, rng, levels, dy=0):
    L = oracle_mod.lib()
    p = oracle_mod.TerrainParams(**TERRAIN)
    g = 1 << levels
    x, z = (int(v) for v in rng.integers(16, g - 16, 2))
    return (float(x), float(L.oracle_terrain_height(p, levels, x, z) + dy), float(z))


def box_voxels(rng, levels, lo, hi, cap=40000):
    g = 1 << levels
    lo = np.clip(np.floor(lo).astype(np.int64) - 2, 0, g - 1)
    hi = np.clip(np.ceil(hi).astype(np.int64) + 2, 0, g - 1)
    n = int(np.prod(hi - lo + 1))
    if n <= cap:
        r = [np.arange(lo[a], hi[a] + 1) for a in range(3)]
        xyz = np.stack(np.meshgrid(*r, indexing="ij"), -1).reshape(-1, 3)
    else:
        xyz = rng.integers(lo, hi + 1, (cap, 3))
    return np.ascontiguousarray(xyz, dtype=np.uint32)


def test_get_value_of_the_oracle_dag_equals_the_reference(oracle_mod, ref_mod):
    rng = np.random.default_rng(3)
    o = oracle_scene(oracle_mod)
    for i in range(6):
        c = surface_centre(oracle_mod, rng, 10)
        o.edit(make_edit(oracle_mod, i % 2, int(rng.integers(0, 16)), c, float(rng.integers(4, 40))))
    ref = ref_mod.RefDag(10, o.export_items())
    xyz = rng.integers(0, 1024, (200000, 3)).astype(np.uint32)
    near = np.array([surface_centre(oracle_mod, rng, 10) for _ in range(200)], dtype=np.int64)
    xyz2 = np.clip(near[:, None, :] + rng.integers(-8, 9, (200, 500, 3)), 0, 1023).reshape(-1, 3).astype(np.uint32)
    for pts in (xyz, xyz2):
        a = o.sample(pts)
        b = ref.get_values(pts)
        assert np.array_equal(a, b)
        assert (b != 0xFFFFFFFF).any() and (b == 0xFFFFFFFF).any()


EDIT_CASES = [
    # tool, radius, centre offset from the surface
    (0, 13.0, 0), (0, 2.5, 3), (1, 21.0, -4), (1, 1.0, 0), (2, 9.0, 2), (2, 0.0, 0), (3, 17.0, -3),
    (4, 19.0, 0), (4, 6.5, -6), (5, 12.0, 0), (5, 7.0, 5), (8, 10.0, 0), (8, 6.0, -2),
]


@pytest.mark.parametrize("case", range(len(EDIT_CASES)))
def test_oracle_edits_equal_the_reference_editors(oracle_mod, ref_mod, case):
    """The voxels of the oracle's DAG after an edit equal, voxel for voxel over the edit's box (and
    around it), the reference editors' decisions evaluated over the DAG before the edit."""
    tool, radius, dy = EDIT_CASES[case]
    rng = np.random.default_rng(100 + case)
    levels = 10
    o = oracle_scene(oracle_mod, levels)
    for i in range(3):  # some history first, so that the edit meets earlier edits' structure
        c = surface_centre(oracle_mod, rng, levels)
        o.edit(make_edit(oracle_mod, i % 2, int(rng.integers(0, 16)), c, float(rng.integers(6, 30))))
    before = ref_mod.RefDag(levels, o.export_items())
    c = np.array(surface_centre(oracle_mod, rng, levels, dy), dtype=np.float64)
    if case % 2:
        c = c + 0.37  # off-grid centres too
    kw = {}
    lo, hi = c - radius - 1, c + radius + 1
    if tool == 5:
        src = c
        dst = c + np.array([float(rng.integers(-40, 41)), 15.0, float(rng.integers(-40, 41))])  # ground into the air
        kw = dict(src=src, dst=dst)
        lo, hi = dst - radius - 1, dst + radius + 1
    if tool == 8:
        kw = dict(threshold=int(rng.integers(8, 18)))
    e = make_edit(oracle_mod, tool, int(rng.integers(0, 16)), c, radius, **kw)
    st = o.edit(e)
    assert st.status == 0
    xyz = box_voxels(rng, levels, lo, hi)
    want = before.edit_values(e, xyz)
    got = o.sample(xyz)
    bad = np.nonzero(want != got)[0]
    assert len(bad) == 0, (case, xyz[bad[:5]].tolist(), want[bad[:5]].tolist(), got[bad[:5]].tolist())
    assert (want != before.get_values(xyz)).any() or tool in (4, 8)  # the edit changed something
