"""Parity of the slab hash tables against set semantics (hash_table_test.cpp:158-240 pattern):
every added key is found and decodes to itself, keys never added are not found, find_or_add stores
one copy per distinct key."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def node_keys(rng, n):
    """DAG-node keys: child-mask byte with popcount U{1..8}, then that many pointers U[0, 2^28)."""
    pc = rng.integers(1, 9, n)
    words, offs = [], []
    pos = 0
    for p in pc:
        bits = rng.choice(8, size=p, replace=False)
        mask = int(sum(1 << int(b) for b in bits))
        key = [mask] + [int(v) for v in rng.integers(0, 1 << 28, p)]
        offs.append(pos)
        words.extend(key)
        pos += len(key)
    return np.array(words, dtype=np.uint32), np.array(offs, dtype=np.uint32)


def leaf_keys(rng, n):
    words, offs, pos = [], [], 0
    for _ in range(n):
        lo, hi = (int(v) for v in rng.integers(0, 1 << 32, 2, dtype=np.uint64))
        if lo == 0 and hi == 0:
            lo = 1
        cnt = bin(lo).count("1") + bin(hi).count("1")
        nmat = (cnt * 4 + 31) // 32
        key = [lo, hi] + [int(v) for v in rng.integers(0, 1 << 32, nmat, dtype=np.uint64)]
        offs.append(pos)
        words.extend(key)
        pos += len(key)
    return np.array(words, dtype=np.uint32), np.array(offs, dtype=np.uint32)


def dev(a):
    import torch

    return torch.from_numpy(a.view(np.int32)).cuda()


def key_list(words, offs):
    ends = list(offs[1:]) + [len(words)]
    return [tuple(words[o:e]) for o, e in zip(offs, ends)]


@pytest.fixture(scope="module")
def dag(svdag_lib):
    d = svdag_lib.MyGPUHashDAG(10, pool_bytes=1 << 30)
    yield d
    d.free()


@pytest.mark.parametrize("lanes", [1, 2, 4, 8, 16, 32])
@pytest.mark.parametrize("kind", [0, 1])
def test_add_then_find(svdag_lib, dag, lanes, kind):
    import torch

    rng = np.random.default_rng(100 + lanes + 7 * kind)
    n = 20000
    gen = node_keys if kind == 0 else leaf_keys
    words, offs = gen(rng, 2 * n)
    keys = key_list(words, offs)
    # add the first n (each twice: duplicates get their own slot, as the reference's add does)
    ins_w, ins_o = words[: offs[n]], offs[:n]
    tbl = dag.create_table(kind, [37] * 9)  # few buckets: long chains of overflow slabs
    h_ins = torch.empty(n, dtype=torch.int32, device="cuda")
    for _ in range(2):
        tbl.add(dev(ins_w), dev(ins_o), n, len(ins_w), h_ins, lanes=lanes)
    h_find = torch.empty(2 * n, dtype=torch.int32, device="cuda")
    tbl.find(dev(words), dev(offs), 2 * n, len(words), h_find, lanes=lanes)
    out = torch.empty((2 * n, 10), dtype=torch.int32, device="cuda")
    tbl.read(h_find, 2 * n, out)
    dag.sync()
    hf = h_find.cpu().numpy().view(np.uint32)
    got = out.cpu().numpy().view(np.uint32)
    inserted = set(keys[:n])
    for i, k in enumerate(keys):
        if k in inserted:
            assert hf[i] != 0xFFFFFFFF
            assert tuple(got[i][: len(k)]) == k
        else:
            assert hf[i] == 0xFFFFFFFF
    st = tbl.stats()
    assert st.items == 2 * n
    assert st.overflow_slabs > 0


@pytest.mark.parametrize("add_lanes,find_lanes", [(1, 32), (32, 1), (8, 2), (2, 16)])
def test_lane_counts_agree_on_buckets_and_tags(svdag_lib, dag, add_lanes, find_lanes):
    """A key hashed by G cooperating lanes (each lane's word terms combined by a group XOR) lands in
    the bucket and carries the tag of the one-thread hash, so a table filled with one lane count is
    searched with another (the reference's warp == thread hash test, utils_tests.cu:204-233)."""
    import torch

    rng = np.random.default_rng(300 + add_lanes * 40 + find_lanes)
    n = 8000
    for kind, gen in ((0, node_keys), (1, leaf_keys)):
        words, offs = gen(rng, 2 * n)
        keys = key_list(words, offs)
        tbl = dag.create_table(kind, [97] * 9)
        h = torch.empty(2 * n, dtype=torch.int32, device="cuda")
        tbl.add(dev(words[: offs[n]]), dev(offs[:n]), n, int(offs[n]), h, lanes=add_lanes)
        tbl.find(dev(words), dev(offs), 2 * n, len(words), h, lanes=find_lanes)
        out = torch.empty((2 * n, 10), dtype=torch.int32, device="cuda")
        tbl.read(h, 2 * n, out)
        dag.sync()
        hf, got = h.cpu().numpy().view(np.uint32), out.cpu().numpy().view(np.uint32)
        assert np.all(hf[:n] != 0xFFFFFFFF)
        assert all(tuple(got[i][: len(keys[i])]) == keys[i] for i in range(n))
        inserted = set(keys[:n])
        assert all(hf[i] == 0xFFFFFFFF for i in range(n, 2 * n) if keys[i] not in inserted)
        tbl.destroy()


@pytest.mark.parametrize("lanes", [1, 8, 32])
def test_find_or_add_dedups(svdag_lib, dag, lanes):
    import torch

    rng = np.random.default_rng(11 + lanes)
    n = 30000
    words, offs = node_keys(rng, n)
    keys = key_list(words, offs)
    # every key twice, shuffled
    order = rng.permutation(np.concatenate([np.arange(n), np.arange(n)]))
    w2, o2, pos = [], [], 0
    for i in order:
        o2.append(pos)
        w2.extend(keys[i])
        pos += len(keys[i])
    w2, o2 = np.array(w2, dtype=np.uint32), np.array(o2, dtype=np.uint32)
    tbl = dag.create_table(0, [500] * 9)
    h = torch.empty(2 * n, dtype=torch.int32, device="cuda")
    tbl.find_or_add(dev(w2), dev(o2), 2 * n, len(w2), h, lanes=lanes)
    out = torch.empty((2 * n, 10), dtype=torch.int32, device="cuda")
    tbl.read(h, 2 * n, out)
    dag.sync()
    hh = h.cpu().numpy().view(np.uint32)
    got = out.cpu().numpy().view(np.uint32)
    first = {}
    for j, i in enumerate(order):
        k = keys[i]
        assert tuple(got[j][: len(k)]) == k
        if k in first:
            assert first[k] == hh[j]
        first[k] = hh[j]
    assert tbl.stats().items == n
    # a second pass finds everything and adds nothing
    tbl.find_or_add(dev(w2), dev(o2), 2 * n, len(w2), h, lanes=lanes)
    dag.sync()
    assert tbl.stats().items == n
    assert np.array_equal(h.cpu().numpy().view(np.uint32), hh)
