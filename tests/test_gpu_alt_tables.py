"""The alternative table layouts on the GPU, thread-per-key and warp-hybrid, through the C ABI.

Same set semantics as tests/test_alt_tables_cpu.py (the reference's hash_table_test.cpp:158-240 and
the verification of extras/hashmap_bench/src/main.cu:640-700): every add gets its own slot,
duplicates included; added keys are found and read back as themselves; keys never added are not
found; exhausting the reserved overflow slabs latches SVDAG_ERR_OOM and stores nothing beyond them.
The file sorts after the other GPU tests so that they run first.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TB, A64, ACC, IC = 1, 2, 3, 4
INVALID = 0xFFFFFFFF


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint32)


def unique_keys(rng, n, k, exclude=None):
    keys = rng.integers(0, 1 << 32, (2 * n + 16, k), dtype=np.uint64).astype(np.uint32)
    if k >= 2:
        keys = keys[(keys[:, 0] != 0) | (keys[:, 1] != 0)]
    keys = np.unique(keys, axis=0)
    if exclude is not None:
        ex = {tuple(r) for r in exclude}
        keys = np.array([r for r in keys if tuple(r) not in ex], dtype=np.uint32).reshape(-1, k)
    keys = keys[rng.permutation(len(keys))[:n]]
    assert len(keys) == n
    return keys


@pytest.fixture(scope="module")
def dag(svdag_lib):
    d = svdag_lib.MyGPUHashDAG(6, pool_bytes=64 << 20, scratch_bytes=16 << 20)
    yield d
    d.free()


@pytest.mark.parametrize("lanes", [1, 32])
@pytest.mark.parametrize("buckets", [7, 1000])
@pytest.mark.parametrize("layout,k", [(TB, 1), (TB, 2), (TB, 5), (A64, 2), (A64, 3), (A64, 9), (ACC, 1), (ACC, 2),
                                      (ACC, 7), (TB, 32), (A64, 32), (ACC, 32), (IC, 1), (IC, 3), (IC, 32)])
def test_add_find_read(svdag_lib, dag, layout, k, buckets, lanes):
    import torch

    rng = np.random.default_rng(1000 * layout + 10 * k + lanes + buckets)
    n = 20000
    keys = unique_keys(rng, n, k)
    ins = keys[rng.permutation(np.concatenate([np.arange(n), np.arange(n)]))]
    t = svdag_lib.AltHashTable(dag, layout, k, buckets, 3 * n)
    try:
        h = torch.empty(2 * n, dtype=torch.int32, device="cuda")
        t.add(dev(ins), 2 * n, h, lanes=lanes)
        t.sync()
        hh = host(h)
        assert np.all(hh != INVALID) and len(np.unique(hh)) == 2 * n
        words = torch.empty((2 * n, k), dtype=torch.int32, device="cuda")
        t.read(h, 2 * n, words)
        assert np.array_equal(host(words), ins)
        st = t.stats()
        assert st.items == 2 * n and st.buckets == buckets
        assert layout != IC or st.overflow_slabs == 0
        absent = unique_keys(rng, n, k, exclude=keys)
        q = np.concatenate([keys, absent])
        f = torch.empty(2 * n, dtype=torch.int32, device="cuda")
        t.find(dev(q), 2 * n, f, lanes=lanes)
        t.read(f, 2 * n, words)
        t.sync()
        fh, got = host(f), host(words)
        assert np.all(fh[:n] != INVALID) and np.all(fh[n:] == INVALID)
        assert np.array_equal(got[:n], keys) and np.all(got[n:] == 0)
    finally:
        t.destroy()


@pytest.mark.parametrize("lanes", [1, 32])
@pytest.mark.parametrize("layout", [TB, A64, ACC, IC])
def test_exhausted_overflow_latches_oom(svdag_lib, dag, layout, lanes):
    import torch

    rng = np.random.default_rng(50 + layout + lanes)
    keys = unique_keys(rng, 2000, 3)
    t = svdag_lib.AltHashTable(dag, layout, 3, 1, 64)
    try:
        h = torch.empty(2000, dtype=torch.int32, device="cuda")
        t.add(dev(keys), 2000, h, lanes=lanes)
        with pytest.raises(svdag_lib.SvdagError) as e:
            t.sync()
        assert e.value.status == 2  # SVDAG_ERR_OOM
        ok = host(h) != INVALID
        if layout == IC:
            assert ok.sum() == 64
        else:
            slots = 32 if layout == TB else 31
            assert ok.sum() == (1 + -(-64 // slots)) * slots
        f = torch.empty(2000, dtype=torch.int32, device="cuda")
        t.find(dev(keys), 2000, f, lanes=lanes)
        t.sync()
        assert np.array_equal(host(f) != INVALID, ok)
    finally:
        t.destroy()


@pytest.mark.parametrize("lanes", [1, 32])
def test_atomic64_rejects_zero_first_words(svdag_lib, dag, lanes):
    import torch

    t = svdag_lib.AltHashTable(dag, A64, 3, 4, 0)
    try:
        h = torch.empty(3, dtype=torch.int32, device="cuda")
        t.add(dev(np.array([[0, 0, 5], [0, 1, 5], [1, 0, 5]])), 3, h, lanes=lanes)
        with pytest.raises(svdag_lib.SvdagError) as e:
            t.sync()
        assert e.value.status == 1  # SVDAG_ERR_INVALID
        hh = host(h)
        assert hh[0] == INVALID and hh[1] != INVALID and hh[2] != INVALID
    finally:
        t.destroy()


def test_hashmap_benchmark_shape(svdag_lib, dag):
    """The reference benchmark's flow at a reduced size: items of 2 words, an initial bulk add,
    searches at hit rates 0..100 %, a second bulk add, then every key of both adds is found."""
    import torch

    rng = np.random.default_rng(9)
    n0, n1, ns = 1 << 16, 1 << 13, 1 << 13
    allk = unique_keys(rng, n0 + n1 + ns, 2)
    init, more, never = allk[:n0], allk[n0:n0 + n1], allk[n0 + n1:]
    for layout in (TB, A64, ACC, IC):
        t = svdag_lib.AltHashTable(dag, layout, 2, (n0 + n1) // 64 + 1, 2 * (n0 + n1))
        try:
            h = torch.empty(n0, dtype=torch.int32, device="cuda")
            t.add(dev(init), n0, h)
            f = torch.empty(ns, dtype=torch.int32, device="cuda")
            for pct in (0, 25, 50, 75, 100):
                hits = ns * pct // 100
                q = np.concatenate([init[rng.permutation(n0)[:hits]], never[:ns - hits]])
                t.find(dev(q), ns, f)
                t.sync()
                assert int((host(f) != INVALID).sum()) == hits
            h1 = torch.empty(n1, dtype=torch.int32, device="cuda")
            t.add(dev(more), n1, h1)
            g = torch.empty(n0 + n1, dtype=torch.int32, device="cuda")
            t.find(dev(np.concatenate([init, more])), n0 + n1, g)
            t.sync()
            assert np.all(host(g) != INVALID)
        finally:
            t.destroy()


@pytest.mark.parametrize("k", [1, 3])
def test_tune_picks_the_fastest_measured_candidate(svdag_lib, dag, k):
    import torch

    rng = np.random.default_rng(70 + k)
    n = 1 << 15
    keys = unique_keys(rng, n, k)
    best, every = svdag_lib.alt_table_tune(dag, dev(keys), n, k)
    assert [(c.layout, c.lanes) for c in every] == [(1, 1), (1, 32), (2, 1), (2, 32), (3, 1), (3, 32), (4, 1)]
    measured = [c for c in every if c.add_ms >= 0]
    # Atomic64 needs two words per item
    assert len(measured) == (5 if k == 1 else 7)
    assert all(c.find_ms >= 0 for c in measured)
    assert min(c.add_ms + c.find_ms for c in measured) == best.add_ms + best.find_ms
    t = svdag_lib.AltHashTable(dag, best.layout, k, n // 64 + 1, 2 * n)
    try:
        h = torch.empty(n, dtype=torch.int32, device="cuda")
        t.add(dev(keys), n, h, lanes=best.lanes)
        t.find(dev(keys), n, h, lanes=best.lanes)
        t.sync()
        assert np.all(host(h) != INVALID)
    finally:
        t.destroy()


@pytest.mark.parametrize("add_lanes,find_lanes", [(1, 32), (32, 1)])
@pytest.mark.parametrize("layout", [TB, A64, ACC, IC])
def test_launch_forms_interoperate(svdag_lib, dag, layout, add_lanes, find_lanes):
    """Keys added thread per key are found warp-hybrid and the other way round: both forms hash,
    place and compare alike."""
    import torch

    rng = np.random.default_rng(90 + layout + add_lanes)
    n = 10000
    keys = unique_keys(rng, n, 4)
    absent = unique_keys(rng, n, 4, exclude=keys)
    t = svdag_lib.AltHashTable(dag, layout, 4, 11, 2 * n)
    try:
        h = torch.empty(n, dtype=torch.int32, device="cuda")
        t.add(dev(keys), n, h, lanes=add_lanes)
        f = torch.empty(2 * n, dtype=torch.int32, device="cuda")
        t.find(dev(np.concatenate([keys, absent])), 2 * n, f, lanes=find_lanes)
        t.sync()
        assert np.array_equal(host(f)[:n], host(h)) and np.all(host(f)[n:] == INVALID)
    finally:
        t.destroy()


@pytest.mark.parametrize("layout", [TB, A64, ACC, IC])
def test_delete_frees_unmarked_items_and_keeps_handles(svdag_lib, dag, layout):
    """The reference's "GPUHashTable Delete GPU" case (hash_table_test.cpp:306-346): 1024 + 512
    items of 2 words added warp-hybrid into 64 buckets, the first 1024 marked active on the GPU,
    freeInactiveItems frees the other 512; kept items are found at their handles, freed ones not at
    all, and adding the freed items again fits them into the slots they left."""
    import torch

    rng = np.random.default_rng(500 + layout)
    n_keep, n_drop = 1024, 512
    for _ in range(10):
        items = unique_keys(rng, n_keep + n_drop, 2)
        t = svdag_lib.AltHashTable(dag, layout, 2, 64, 2 * (n_keep + n_drop))
        try:
            h = torch.empty(n_keep + n_drop, dtype=torch.int32, device="cuda")
            t.add(dev(items), n_keep + n_drop, h, lanes=32)
            t.clearActiveFlags()
            t.markAsActive(h[:n_keep], n_keep)
            assert t.freeInactiveItems() == n_drop
            assert t.stats().items == n_keep
            f = torch.empty(n_keep + n_drop, dtype=torch.int32, device="cuda")
            t.find(dev(items), n_keep + n_drop, f)
            t.sync()
            hf = host(f)
            assert np.array_equal(hf[:n_keep], host(h)[:n_keep]) and np.all(hf[n_keep:] == INVALID)
            slabs = t.stats().overflow_slabs
            g = torch.empty(n_drop, dtype=torch.int32, device="cuda")
            t.add(dev(items[n_keep:]), n_drop, g)
            t.find(dev(items), n_keep + n_drop, f)
            t.sync()
            assert np.all(host(f) != INVALID) and np.array_equal(host(f)[n_keep:], host(g))
            assert t.stats().items == n_keep + n_drop and t.stats().overflow_slabs == slabs
        finally:
            t.destroy()
