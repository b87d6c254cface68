"""The reference's own DAG file (MyGPUHashDAG::writeTo / readFrom, version 3) on the host: the
library's writer and reader (svdag_items_to_v3, svdag_v3_to_items) round-trip DAGs, lay every item
where the reference's tables look for it, and reject damaged files.

The layout checks parse the file here independently, following the reference's serialisation
(binary_writer.h:84-116, array.h:30-53 and 311-315, gpu_hash_table_base.cu:117-137,
dynamic_slab_alloc.cu:172-179) and its table addressing (gpu_hash_table_base.h:310-321,
compact_acceleration_hash_table.h:478-531, dynamic_slab_alloc.h:355-369, my_gpu_base_dag.h:334-342).
The reference's own code reading and writing these files is checked on a GPU box
(tests/test_gpu_v3.py), where its host DAG can run.
"""
import numpy as np
import pytest

from snapshot_util import same_dag, snap_parts, snapshot_from_rows
from test_io import build_basic_dag, random_grid


def xor_hash(words):
    """Utils::xorHash32xN (utils.h:395-403)."""
    seed = 0
    for i, w in enumerate(words):
        seed ^= ((2717583853 * int(w) + i * 1117415409) & 0xFFFFFFFF) % 4294967291
    return seed


def tag(words):
    """computeAccelerationHash (compact_acceleration_hash_table.h:478-489)."""
    t = 0
    for i, w in enumerate(words):
        t ^= ((32 - i) * int(w)) & 0xFFFFFFFF
    t &= 0xFF
    return t or 1


class V3File:
    """Independent parse of a version-3 file; records the byte offset of every memory-type field."""

    def __init__(self, path):
        self.b = np.fromfile(path, np.uint8)
        self.at = 0
        self.mem_offsets, self.mem_kinds = [], []
        assert self.u32() == 3
        n = self.u64()
        self.mem()
        self.ff = self.words(n)
        self.width, self.height = self.u32(), self.u32()
        self.root = self.u32()
        assert self.u64() == 9
        self.mem()
        self.tables = []
        for t in range(9):
            size, slab, buckets = self.u32(), self.u32(), self.u32()
            n = self.u32()
            self.mem()
            first = self.words(n).reshape(buckets, slab)
            unit, superw = self.u32(), self.u32()
            nsuper = self.u64()
            self.mem("super block list")
            supers = []
            for _ in range(nsuper):
                assert self.u64() == superw
                self.mem()
                supers.append(self.words(superw))
            assert self.u64() == nsuper
            units, items, slabs = self.u32(), self.u32(), self.u32()
            self.tables.append(dict(size=size, slab=slab, buckets=buckets, first=first, unit=unit, superw=superw,
                                    supers=supers, units=units))
        assert self.at == len(self.b)

    def take(self, n):
        v = self.b[self.at: self.at + n]
        assert len(v) == n, "truncated"
        self.at += n
        return v

    def u32(self):
        return int(self.take(4).view("<u4")[0])

    def u64(self):
        return int(self.take(8).view("<u8")[0])

    def words(self, n):
        return self.take(4 * n).view("<u4")

    def mem(self, kind="array"):
        self.mem_offsets.append(self.at)
        self.mem_kinds.append(kind)
        v = self.u32()
        assert v < 4
        return v

    def slab_of(self, t, ptr):
        """(slab words, slot, bucket or None) of an item pointer."""
        T = self.tables[t]
        slot, slab = ptr & 31, ptr >> 6
        if ptr >> 5 & 1:
            return T["first"][slab], slot, slab
        sb, unit = slab // 16384, slab % 16384
        sup = T["supers"][sb]
        assert sup[unit >> 5] >> (unit & 31) & 1, "unit not allocated"
        return sup[512 + unit * T["slab"]: 512 + (unit + 1) * T["slab"]], slot, None

    def item(self, handle, leaf):
        size = (handle >> 29) + (3 if leaf else 2)
        t = size - 2
        s, slot, _ = self.slab_of(t, handle & ((1 << 29) - 1))
        assert s[slot >> 2] >> ((slot & 3) * 8) & 0xFF, "empty slot"
        return s[10 + slot * size: 10 + (slot + 1) * size], t

    def bucket_chain(self, t, bucket):
        """Pointers of the slabs chained from a bucket's first slab."""
        T = self.tables[t]
        s = T["first"][bucket]
        out = []
        while int(s[8]) != 0xFFFFFFFF:
            p = int(s[8])
            out.append(p)
            s, _, _ = self.slab_of(t, p << 6)
        return out


def oracle_snapshot(svdag, oracle_mod, levels):
    """A DAG with materials, fully-filled regions, paint and a hole, built by the oracle."""
    o = oracle_mod.OracleDag(levels)
    g = 1 << levels
    for tool, mat, c, r in [(2, 7, (g * 0.3, g * 0.3, g * 0.3), g * 0.2), (0, 3, (g * 0.55, g * 0.5, g * 0.5), g * 0.3),
                            (4, 11, (g * 0.6, g * 0.6, g * 0.4), g * 0.15), (1, 0, (g * 0.5, g * 0.45, g * 0.55), g * 0.1)]:
        e = oracle_mod.Edit()
        e.tool, e.material, e.radius = tool, mat, r
        e.center[:] = list(c)
        assert o.edit(e).status == 0
    return snapshot_from_rows(svdag, levels, o.export_items()), o


@pytest.mark.parametrize("levels", [4, 6, 8])
def test_round_trip_basic_dags(svdag_lib, tmp_path, levels):
    data = build_basic_dag(random_grid(np.random.default_rng(levels), levels), levels)
    snap = svdag_lib.basic_dag_to_items(data, levels, 5)
    p = str(tmp_path / "dag.v3")
    svdag_lib.items_to_v3(snap, p, svdag_lib.V3_CPU)
    back = svdag_lib.v3_to_items(p, levels)
    assert same_dag(levels, snap_parts(snap), snap_parts(back))


def test_round_trip_and_layout_of_an_edited_dag(svdag_lib, oracle_mod, tmp_path):
    levels = 9
    snap, o = oracle_snapshot(svdag_lib, oracle_mod, levels)
    p = str(tmp_path / "dag.v3")
    svdag_lib.items_to_v3(snap, p, svdag_lib.V3_CPU)
    back = svdag_lib.v3_to_items(p, levels)
    assert same_dag(levels, snap_parts(snap), snap_parts(back))

    f = V3File(p)
    LL = levels - 2
    assert (f.width, f.height) == (levels, 16)
    assert all(m == 3 for m in (int(f.b[o]) for o in f.mem_offsets[:3]))
    for t, T in enumerate(f.tables):
        assert T["size"] == t + 2 and T["slab"] == 10 + 32 * (t + 2) and T["unit"] == T["slab"]
        assert T["superw"] == 512 + 16384 * T["slab"]
    # every reachable item: in the bucket its hash names (its own slab or one chained from it),
    # under the tag of its words; children resolve at the level below
    seen = 0
    frontier = {f.root}
    for level in range(LL + 1):
        nxt = set()
        for h in frontier:
            w, t = f.item(h, level == LL)
            ptr = h & ((1 << 29) - 1)
            _, slot, first_bucket = f.slab_of(t, ptr)
            bucket = xor_hash(w) % f.tables[t]["buckets"]
            if first_bucket is not None:
                assert first_bucket == bucket
            else:
                assert ptr >> 6 in f.bucket_chain(t, bucket)
            s, _, _ = f.slab_of(t, ptr)
            assert s[slot >> 2] >> ((slot & 3) * 8) & 0xFF == tag(w)
            if level < LL:
                nxt.update(int(c) for c in w[1:])
            seen += 1
        frontier = nxt
    assert seen == int(snap.level_items.sum())
    # the fully-filled items of every level and material
    for m in range(16):
        leaf, _ = f.item(int(f.ff[m * levels + LL]), True)
        assert list(leaf) == [0xFFFFFFFF, 0xFFFFFFFF] + [m * 0x11111111] * 8
        for level in range(LL - 1, -1, -1):
            node, _ = f.item(int(f.ff[m * levels + level]), False)
            assert int(node[0]) == 0xFF | 1 << 8 | m << 9
            assert all(int(c) == int(f.ff[m * levels + level + 1]) for c in node[1:])
    # values through the file equal the oracle's
    rng = np.random.default_rng(0)
    xyz = rng.integers(0, 1 << levels, (2000, 3)).astype(np.uint32)
    want = o.sample(xyz)
    got = []
    for x, y, z in xyz.tolist():
        h, level, v = f.root, 0, 0xFFFFFFFF
        while True:
            if level == LL:
                w, _ = f.item(h, True)
                idx = (((x >> 1 & 1) << 2 | (y >> 1 & 1) << 1 | (z >> 1 & 1)) << 3) | ((x & 1) << 2 | (y & 1) << 1 | (z & 1))
                mask = int(w[0]) | int(w[1]) << 32
                if mask >> idx & 1:
                    k = bin(mask & ((1 << idx) - 1)).count("1")
                    v = int(w[2 + (4 * k) // 32]) >> ((4 * k) % 32) & 0xF
                break
            w, _ = f.item(h, False)
            sh = levels - 1 - level
            c = (x >> sh & 1) << 2 | (y >> sh & 1) << 1 | (z >> sh & 1)
            if not int(w[0]) >> c & 1:
                break
            h = int(w[1 + bin(int(w[0]) & ((1 << c) - 1)).count("1")])
            level += 1
        got.append(v)
    assert np.array_equal(np.array(got, np.uint32), want)


def test_memory_type_fields(svdag_lib, tmp_path):
    """A file for the engine's DAG (GPU_Malloc) differs from a host DAG's file only in its memory-type
    fields; each table's super block list is a host array in both (dynamic_slab_alloc.cu:61)."""
    levels = 6
    snap = svdag_lib.basic_dag_to_items(build_basic_dag(random_grid(np.random.default_rng(2), levels), levels), levels, 1)
    a, b = str(tmp_path / "cpu.v3"), str(tmp_path / "gpu.v3")
    svdag_lib.items_to_v3(snap, a, svdag_lib.V3_CPU)
    svdag_lib.items_to_v3(snap, b, svdag_lib.V3_GPU_MALLOC)
    fa, fb = V3File(a), V3File(b)
    assert fa.mem_offsets == fb.mem_offsets and len(fa.b) == len(fb.b)
    assert set(np.nonzero(fa.b != fb.b)[0].tolist()) <= set(fa.mem_offsets)
    for off, kind in zip(fa.mem_offsets, fa.mem_kinds):
        assert int(fa.b[off]) == 3
        assert int(fb.b[off]) == (3 if kind == "super block list" else 1)


def test_empty_dag(svdag_lib, tmp_path):
    levels = 5
    nl = levels - 1
    empty = svdag_lib.ItemSnapshot(levels, np.zeros(0, np.uint32), np.zeros(nl, np.uint64), np.zeros(nl, np.uint64))
    p = str(tmp_path / "empty.v3")
    svdag_lib.items_to_v3(empty, p, svdag_lib.V3_CPU)
    assert V3File(p).root == 0xFFFFFFFF
    back = svdag_lib.v3_to_items(p, levels)
    assert int(back.level_items.sum()) == 0 and len(back.words) == 0


def test_damaged_files_are_rejected(svdag_lib, tmp_path):
    levels = 6
    snap = svdag_lib.basic_dag_to_items(build_basic_dag(random_grid(np.random.default_rng(3), levels), levels), levels, 2)
    p = str(tmp_path / "dag.v3")
    svdag_lib.items_to_v3(snap, p, svdag_lib.V3_CPU)
    good = np.fromfile(p, np.uint8)
    f = V3File(p)

    def status(data, lv=levels):
        q = str(tmp_path / "bad.v3")
        data.tofile(q)
        with pytest.raises(svdag_lib.SvdagError) as e:
            svdag_lib.v3_to_items(q, lv)
        return e.value.status

    assert status(good[: len(good) // 2]) == 4  # truncated
    bad = good.copy()
    bad[:4] = np.frombuffer(np.uint32(4).tobytes(), np.uint8)  # another version
    assert status(bad) == 7
    assert status(good, levels + 1) == 1  # another scene depth
    # the root's slot marked empty
    root = f.root
    s, slot, _ = f.slab_of(root >> 29, root & ((1 << 29) - 1))
    byte = s.ctypes.data - f.b.ctypes.data + 4 * (slot >> 2) + (slot & 3)
    bad = good.copy()
    assert bad[byte] != 0
    bad[byte] = 0
    assert status(bad) == 4
    # a root handle naming an allocator unit that was never allocated
    root_at = 4 + 8 + 4 + 4 * levels * 16 + 8
    bad = good.copy()
    bad[root_at: root_at + 4] = np.frombuffer(np.uint32((root & 0xE0000000) | 0x3FFFF << 6).tobytes(), np.uint8)
    assert status(bad) == 4
    # a root handle whose size field disagrees with the item's child count
    size_bits = root >> 29
    bad = good.copy()
    bad[root_at: root_at + 4] = np.frombuffer(np.uint32((root & 0x1FFFFFFF) | ((size_bits + 1) % 8) << 29).tobytes(), np.uint8)
    assert status(bad) == 4


def test_snapshot_that_does_not_parse(svdag_lib, tmp_path):
    levels = 5
    snap = svdag_lib.basic_dag_to_items(build_basic_dag(random_grid(np.random.default_rng(5), levels), levels), levels, 2)
    bad = svdag_lib.ItemSnapshot(levels, snap.words.copy(), snap.level_words.copy(), snap.level_items.copy())
    bad.words[1] = 1 << 30  # a child ordinal of the root out of range
    with pytest.raises(svdag_lib.SvdagError) as e:
        svdag_lib.items_to_v3(bad, str(tmp_path / "x.v3"), svdag_lib.V3_CPU)
    assert e.value.status == 1


def test_corrupted_files_never_crash_the_reader(svdag_lib, tmp_path):
    """Random byte changes anywhere in a file: the reader returns a status or a snapshot that parses;
    it never reads outside the buffer (the buffer is exactly the file, no slack)."""
    import ctypes as C

    levels = 6
    snap = svdag_lib.basic_dag_to_items(build_basic_dag(random_grid(np.random.default_rng(8), levels), levels), levels, 4)
    p = str(tmp_path / "dag.v3")
    svdag_lib.items_to_v3(snap, p, svdag_lib.V3_CPU)
    good = np.fromfile(p, np.uint8)
    f = V3File(p)
    # the bytes that matter most: headers, the fully-filled array, the root, the first slabs' tags and
    # items; and anywhere at all
    hot = list(range(0, 4 + 8 + 4 + 4 * levels * 16 + 16 + 12 + 8))
    for T in f.tables:
        base = T["first"].ctypes.data - f.b.ctypes.data
        hot += list(range(base, base + min(T["first"].nbytes, 512)))
    rng = np.random.default_rng(9)
    L = svdag_lib.lib()
    nl = levels - 1
    lw, li, total = np.zeros(nl, np.uint64), np.zeros(nl, np.uint64), C.c_uint64()
    statuses = set()
    rewritten = 0
    for trial in range(80):
        bad = good.copy()
        where = rng.choice(hot, 3) if trial % 2 == 0 else rng.integers(0, len(bad), 3)
        for w_ in where:
            bad[int(w_)] = rng.integers(0, 256)
        cut = len(bad) if trial % 5 else int(rng.integers(0, len(bad)))
        buf = np.ascontiguousarray(bad[:cut])
        st = L.svdag_v3_to_items(buf.ctypes.data if cut else None, cut, levels, None, 0, lw.ctypes.data, li.ctypes.data,
                                 C.byref(total))
        statuses.add(int(st))
        if st in (0, 2):  # a snapshot came out: it must be one the loader accepts
            words = np.zeros(max(total.value, 1), np.uint32)
            assert L.svdag_v3_to_items(buf.ctypes.data, cut, levels, words.ctypes.data, len(words), lw.ctypes.data,
                                       li.ctypes.data, C.byref(total)) == 0
            if rewritten < 2:
                back = svdag_lib.ItemSnapshot(levels, words[: total.value], lw.copy(), li.copy())
                svdag_lib.items_to_v3(back, str(tmp_path / "re.v3"), svdag_lib.V3_CPU)
                rewritten += 1
    assert statuses - {0, 1, 2, 4, 7} == set()
    assert 4 in statuses
