"""Child process of tests/test_alt_tables_cpu.py: runs the warp-hybrid add and find of the alternative
table layouts on emulated warps (tests/alt_tables_host.cpp) and checks their set semantics. A child,
because the emulator aborts the process when a lane misses a warp collective.

usage: python alt_warp_child.py <host .so> <layout> <item words> <buckets> <warps>
"""
import ctypes as C
import sys

import numpy as np

INVALID = 0xFFFFFFFF
ERR_INVALID, ERR_OOM = 1, 2


def load(so):
    lib = C.CDLL(so)
    lib.alt_host_create.restype = C.c_void_p
    lib.alt_host_create.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64]
    lib.alt_host_destroy.argtypes = [C.c_void_p]
    lib.alt_host_warp_op.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_int]
    lib.alt_host_find.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]
    lib.alt_host_read.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    lib.alt_host_status.restype = C.c_uint32
    lib.alt_host_status.argtypes = [C.c_void_p]
    lib.alt_host_stats.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.alt_host_linked_overflow.restype = C.c_uint64
    lib.alt_host_linked_overflow.argtypes = [C.c_void_p]
    return lib


def unique_keys(rng, n, k, exclude=()):
    ex = {tuple(r) for r in exclude}
    out, seen = [], set()
    while len(out) < n:
        r = tuple(int(v) for v in rng.integers(0, 1 << 32, k, dtype=np.uint64))
        if (k >= 2 and r[0] == 0 and r[1] == 0) or r in seen or r in ex:
            continue
        seen.add(r)
        out.append(r)
    return np.array(out, dtype=np.uint32).reshape(n, k)


class Table:
    def __init__(self, lib, layout, k, buckets, reserved, warps):
        self.lib, self.k, self.warps = lib, k, warps
        self.h = lib.alt_host_create(layout, k, buckets, reserved)
        assert self.h

    def op(self, keys, add):
        keys = np.ascontiguousarray(keys, dtype=np.uint32)
        out = np.full(len(keys), 0x12345678, dtype=np.uint32)
        self.lib.alt_host_warp_op(self.h, keys.ctypes.data, len(keys), out.ctypes.data, self.warps, 1 if add else 0)
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


def main():
    so, layout, k, buckets, warps = sys.argv[1], *(int(v) for v in sys.argv[2:6])
    lib = load(so)
    rng = np.random.default_rng(layout * 1000 + k * 10 + buckets + warps)
    n = 500
    keys = unique_keys(rng, n, k)
    ins = keys[rng.permutation(np.concatenate([np.arange(n), np.arange(n)]))]
    # every key twice; 1000 keys is not a multiple of 32, so the last warp has idle lanes
    t = Table(lib, layout, k, buckets, 3 * n, warps)
    try:
        h = t.op(ins, add=True)
        assert t.status() == 0, t.status()
        assert np.all(h != INVALID) and len(np.unique(h)) == 2 * n, "two adds got the same slot"
        assert np.array_equal(t.read(h), ins)
        items, overflow = t.stats()
        assert items == 2 * n, items
        assert lib.alt_host_linked_overflow(t.h) == overflow
        absent = unique_keys(rng, n, k, exclude=keys)
        f = t.op(np.concatenate([keys, absent]), add=False)
        assert np.all(f[:n] != INVALID) and np.all(f[n:] == INVALID)
        assert np.array_equal(t.read(f[:n]), keys)
        # the thread-per-key find agrees with the warp-hybrid one (same hash, same slot order)
        q = np.ascontiguousarray(np.concatenate([keys, absent]), dtype=np.uint32)
        g = np.empty(2 * n, dtype=np.uint32)
        lib.alt_host_find(t.h, q.ctypes.data, 2 * n, g.ctypes.data, 8)
        assert np.array_equal(g, f)
        assert t.status() == 0
    finally:
        t.free()
    # exhaustion: one bucket slab and ceil(64 / slots) overflow slabs, every slot used, nothing beyond
    more = unique_keys(rng, 300, k)
    t = Table(lib, layout, k, 1, 64, warps)
    try:
        h = t.op(more, add=True)
        assert t.status() == ERR_OOM, t.status()
        ok = h != INVALID
        slots = 32 if layout == 1 else 31
        assert ok.sum() == (1 + -(-64 // slots)) * slots, int(ok.sum())
        assert np.array_equal(t.read(h[ok]), more[ok])
        f = t.op(more, add=False)
        assert np.array_equal(f != INVALID, ok)
    finally:
        t.free()
    if layout == 2 and k == 3:
        t = Table(lib, layout, k, 4, 0, 1)
        try:
            h = t.op(np.array([[0, 0, 5], [0, 1, 5], [1, 0, 5]], np.uint32), add=True)
            assert h[0] == INVALID and h[1] != INVALID and h[2] != INVALID
            assert t.status() == ERR_INVALID
        finally:
            t.free()
    print("ok")


if __name__ == "__main__":
    main()
