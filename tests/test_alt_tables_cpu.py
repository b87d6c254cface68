"""The alternative table layouts' claim, chain and lookup logic on the CPU.

`tests/alt_tables_host.cpp` compiles the library's layout header (svdag_alt_tables.cuh) for the host,
unchanged, and drives its thread-per-key add and find from several threads at once. The checks are the
set semantics of the reference's table tests (hash_table_test.cpp:158-240) and of its table benchmark's
verification (extras/hashmap_bench/src/main.cu:640-700): every add gets its own slot, duplicates
included; every added key is found and reads back as itself; keys never added are not found.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
TB, A64, ACC, IC = 1, 2, 3, 4
INVALID = 0xFFFFFFFF
ERR_INVALID, ERR_OOM = 1, 2


def _compile(out_dir, extra=()):
    so = os.path.join(out_dir, "alt_tables_host%s.so" % ("_tsan" if extra else ""))
    cmd = ["g++", "-O2", "-std=c++17", "-pthread", "-shared", "-fPIC", *extra, os.path.join(HERE, "alt_tables_host.cpp"),
           "-o", so]
    subprocess.check_call(cmd)
    return so


def _load(so):
    lib = C.CDLL(so)
    lib.alt_host_create.restype = C.c_void_p
    lib.alt_host_create.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64]
    lib.alt_host_destroy.argtypes = [C.c_void_p]
    for f in (lib.alt_host_add, lib.alt_host_find):
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]
    lib.alt_host_read.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    lib.alt_host_status.restype = C.c_uint32
    lib.alt_host_status.argtypes = [C.c_void_p]
    lib.alt_host_stats.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.alt_host_linked_overflow.restype = C.c_uint64
    lib.alt_host_linked_overflow.argtypes = [C.c_void_p]
    lib.alt_host_clear_active.argtypes = [C.c_void_p]
    lib.alt_host_mark_active.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32]
    lib.alt_host_free_inactive.restype = C.c_uint64
    lib.alt_host_free_inactive.argtypes = [C.c_void_p]
    return lib


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    return _load(_compile(str(tmp_path_factory.mktemp("alt"))))


class Table:
    def __init__(self, lib, layout, k, buckets, reserved):
        self.lib, self.k = lib, k
        self.h = lib.alt_host_create(layout, k, buckets, reserved)
        assert self.h

    def add(self, keys, threads=8):
        keys = np.ascontiguousarray(keys, dtype=np.uint32)
        out = np.empty(len(keys), dtype=np.uint32)
        self.lib.alt_host_add(self.h, keys.ctypes.data, len(keys), out.ctypes.data, threads)
        return out

    def find(self, keys, threads=8):
        keys = np.ascontiguousarray(keys, dtype=np.uint32)
        out = np.empty(len(keys), dtype=np.uint32)
        self.lib.alt_host_find(self.h, keys.ctypes.data, len(keys), out.ctypes.data, threads)
        return out

    def read(self, handles):
        handles = np.ascontiguousarray(handles, dtype=np.uint32)
        out = np.empty((len(handles), self.k), dtype=np.uint32)
        self.lib.alt_host_read(self.h, handles.ctypes.data, len(handles), out.ctypes.data)
        return out

    def status(self):
        return int(self.lib.alt_host_status(self.h))

    def stats(self):
        items, overflow = C.c_uint64(), C.c_uint64()
        self.lib.alt_host_stats(self.h, C.byref(items), C.byref(overflow))
        return items.value, overflow.value

    def free(self):
        self.lib.alt_host_destroy(self.h)


def unique_keys(rng, n, k, exclude=None):
    """n distinct random keys of k words; none equal to a row of `exclude`, none with two zero first words."""
    keys = rng.integers(0, 1 << 32, (2 * n + 16, k), dtype=np.uint64).astype(np.uint32)
    if k >= 2:
        keys = keys[(keys[:, 0] != 0) | (keys[:, 1] != 0)]
    rows = {tuple(r) for r in exclude} if exclude is not None else set()
    out, seen = [], set()
    for r in map(tuple, keys):
        if r not in seen and r not in rows:
            seen.add(r)
            out.append(r)
        if len(out) == n:
            break
    return np.array(out, dtype=np.uint32).reshape(n, k)


CASES = [(TB, 1), (TB, 2), (TB, 5), (TB, 32), (A64, 2), (A64, 3), (A64, 9), (A64, 32), (ACC, 1), (ACC, 2), (ACC, 7),
         (ACC, 32), (IC, 1), (IC, 3), (IC, 32)]


@pytest.mark.parametrize("buckets", [5, 300])
@pytest.mark.parametrize("layout,k", CASES)
def test_add_find_read_set_semantics(host, layout, k, buckets):
    rng = np.random.default_rng(layout * 100 + k + buckets)
    n = 3000
    keys = unique_keys(rng, n, k)
    ins = keys[rng.permutation(np.concatenate([np.arange(n), np.arange(n)]))]  # every key twice
    t = Table(host, layout, k, buckets, reserved=4 * n)
    try:
        h = t.add(ins)
        assert t.status() == 0
        assert np.all(h != INVALID)
        assert len(np.unique(h)) == 2 * n, "two adds got the same slot"
        assert np.array_equal(t.read(h), ins)
        items, overflow = t.stats()
        if layout != IC:
            slots = 32 if layout == TB else 31
            assert items == 2 * n and overflow >= -(-2 * n // slots) - buckets
            assert t.lib.alt_host_linked_overflow(t.h) == overflow  # no slab taken and left unlinked
        else:
            assert items == 2 * n and overflow == 0  # every node taken is linked
        absent = unique_keys(rng, n, k, exclude=keys)
        fh = t.find(np.concatenate([keys, absent]))
        assert np.all(fh[:n] != INVALID) and np.all(fh[n:] == INVALID)
        assert np.array_equal(t.read(fh[:n]), keys)
        assert t.status() == 0
    finally:
        t.free()


@pytest.mark.parametrize("layout,k", [(TB, 3), (A64, 3), (ACC, 3), (IC, 3)])
def test_exhausted_overflow_latches_oom(host, layout, k):
    rng = np.random.default_rng(7)
    keys = unique_keys(rng, 400, k)
    t = Table(host, layout, k, 1, reserved=64)  # one bucket slab and ceil(64 / slots) overflow slabs
    try:
        h = t.add(keys)
        assert t.status() == ERR_OOM
        ok = h != INVALID
        if layout == IC:
            assert ok.sum() == 64  # the reserved nodes, nothing beyond
        else:
            slots = 32 if layout == TB else 31
            assert ok.sum() == (1 + -(-64 // slots)) * slots  # every slot of those slabs, nothing beyond
        assert np.array_equal(t.read(h[ok]), keys[ok])
        fh = t.find(keys)
        assert np.all((fh != INVALID) == ok)
    finally:
        t.free()


@pytest.mark.parametrize("layout", [TB, A64, ACC, IC])
def test_delete_frees_unmarked_items_and_keeps_handles(host, layout):
    """The reference's "GPUHashTable Delete" case (hash_table_test.cpp:262-303): 1024 + 512 items
    of 2 words in 64 buckets, the first 1024 marked active, freeInactiveItems frees exactly the 512
    others; every kept item is found at its original handle, any other find decodes to its key. Ten
    random item sets, as GENERATE(take(10, ...)) draws. Freed slots are then reused by new adds."""
    rng = np.random.default_rng(400 + layout)
    n_keep, n_drop = 1024, 512
    for _ in range(10):
        items = unique_keys(rng, n_keep + n_drop, 2)
        t = Table(host, layout, 2, 64, reserved=2 * (n_keep + n_drop))
        try:
            h = t.add(items)
            assert np.all(h != INVALID)
            before = t.stats()[0]
            t.lib.alt_host_clear_active(t.h)
            keep = np.ascontiguousarray(h[:n_keep])
            t.lib.alt_host_mark_active(t.h, keep.ctypes.data, n_keep, 8)
            assert t.lib.alt_host_free_inactive(t.h) == n_drop
            assert t.stats()[0] == before - n_drop
            f = t.find(items)
            assert np.array_equal(f[:n_keep], h[:n_keep])
            found = f != INVALID
            assert np.array_equal(t.read(f[found]), items[found])
            assert not found[n_keep:].any()  # distinct random items: the freed ones are gone
            # adding the freed items again fills exactly the slots they left (same buckets), so the
            # slab layouts need no new slab; IndividualChaining takes fresh nodes. All are found.
            again = np.ascontiguousarray(items[n_keep:])
            taken = t.lib.alt_host_linked_overflow(t.h)
            g = t.add(again)
            assert np.all(g != INVALID) and t.status() == 0
            if layout != IC:
                assert t.lib.alt_host_linked_overflow(t.h) == taken
            assert np.array_equal(t.find(again), g) and np.array_equal(t.find(items[:n_keep]), h[:n_keep])
        finally:
            t.free()


def test_atomic64_rejects_items_with_zero_first_words(host):
    t = Table(host, A64, 3, 4, reserved=0)
    try:
        h = t.add(np.array([[0, 0, 5], [0, 1, 5], [1, 0, 5]], np.uint32), threads=1)
        assert h[0] == INVALID and h[1] != INVALID and h[2] != INVALID
        assert t.status() == ERR_INVALID
        assert t.find(np.array([[0, 0, 5]], np.uint32), threads=1)[0] == INVALID
    finally:
        t.free()


@pytest.mark.parametrize("layout", [TB, A64, ACC, IC])
def test_handles_that_name_no_item_read_as_zeros(host, layout):
    t = Table(host, layout, 4, 3, reserved=31)
    try:
        h = t.add(np.array([[9, 8, 7, 6]], np.uint32), threads=1)
        h0 = int(h[0])
        if layout == IC:  # node ids: the one node taken is 0
            bad = np.array([INVALID, 1, 30, 31, 1 << 30], np.uint32)
        else:
            bad = np.array([INVALID, h0 ^ 1, 3 * 32 + 5, 1 << 30, (h0 & 0xFFFFFFE0) | 31], np.uint32)
        out = t.read(bad)
        assert np.all(out == 0)
        assert np.array_equal(t.read(h), [[9, 8, 7, 6]])
    finally:
        t.free()


def test_concurrent_adds_are_race_free_under_thread_sanitizer(tmp_path):
    """The add phase claims and links with atomics only: ThreadSanitizer finds no data race when 8
    threads fill three buckets' chains at once (run in a child process, where the sanitizer is
    loaded first)."""
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    try:
        so = _compile(str(tmp_path), extra=("-fsanitize=thread", "-g"))
    except (subprocess.CalledProcessError, OSError):
        pytest.skip("no ThreadSanitizer runtime")
    script = f"""
import ctypes as C, numpy as np
lib = C.CDLL({so!r})
lib.alt_host_create.restype = C.c_void_p
lib.alt_host_create.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64]
lib.alt_host_add.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]
lib.alt_host_status.restype = C.c_uint32
lib.alt_host_status.argtypes = [C.c_void_p]
rng = np.random.default_rng(5)
for layout in (1, 2, 3, 4):
    keys = rng.integers(1, 1 << 32, (2000, 3), dtype=np.uint64).astype(np.uint32)
    t = lib.alt_host_create(layout, 3, 3, 4000)
    out = np.empty(2000, np.uint32)
    lib.alt_host_add(t, keys.ctypes.data, 2000, out.ctypes.data, 8)
    assert lib.alt_host_status(t) == 0 and len(set(out.tolist())) == 2000
print("ok")
"""
    rt = subprocess.run(["g++", "-print-file-name=libtsan.so"], capture_output=True, text=True).stdout.strip()
    if not os.path.isabs(rt) or not os.path.exists(rt):
        pytest.skip("no ThreadSanitizer runtime")
    env = dict(os.environ, LD_PRELOAD=rt, TSAN_OPTIONS="halt_on_error=1 exitcode=66 report_signal_unsafe=0")
    r = subprocess.run(["python", "-c", script], capture_output=True, text=True, env=env, timeout=600)
    if r.returncode != 0 and "ThreadSanitizer" not in r.stderr and "ok" not in r.stdout:
        pytest.skip("ThreadSanitizer could not run here: " + r.stderr[-300:])
    assert "WARNING: ThreadSanitizer" not in r.stderr, r.stderr[-3000:]
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr[-2000:]


@pytest.fixture(scope="module")
def host_so(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    return _compile(str(tmp_path_factory.mktemp("altw")))


@pytest.mark.parametrize("warps", [1, 4])
@pytest.mark.parametrize("layout,k,buckets", [(TB, 1, 5), (TB, 3, 40), (TB, 32, 5), (A64, 2, 5), (A64, 3, 40),
                                              (A64, 32, 5), (ACC, 1, 5), (ACC, 3, 40), (ACC, 32, 5)])
def test_warp_hybrid_forms_on_emulated_warps(host_so, layout, k, buckets, warps):
    """The warp-hybrid add and find (the lanes = 32 kernels) run by emulated warps of 32 threads,
    several warps at once: same set semantics, exact exhaustion and no lane missing a collective."""
    r = subprocess.run(["python", os.path.join(HERE, "alt_warp_child.py"), host_so, str(layout), str(k), str(buckets),
                        str(warps)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), (r.stdout[-1000:], r.stderr[-3000:])
