"""The allocation-free find-or-add gives the same results as the arena-backed one.

svdag_table_find_or_add_static exists for callers that must not allocate GPU memory while they run
(for example code recording a CUDA graph, or a real-time loop that may not reach the allocator); its
scratch is a fixed array inside the library. This file is collected last so that a run stopping at the
first failure has already run every other test; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_KEYS = 65536


def node_keys(rng, n):
    pc = rng.integers(1, 9, n)
    keys = []
    for p in pc:
        bits = rng.choice(8, size=p, replace=False)
        keys.append((int(sum(1 << int(b) for b in bits)),) + tuple(int(v) for v in rng.integers(0, 1 << 28, p)))
    return keys


def pack(keys):
    words, offs, pos = [], [], 0
    for k in keys:
        offs.append(pos)
        words.extend(k)
        pos += len(k)
    return np.array(words, dtype=np.uint32), np.array(offs, dtype=np.uint32)


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def labels(h):
    """Partition of the batch by handle, labelled by each handle's first position (table independent)."""
    first = {}
    return np.array([first.setdefault(int(v), i) for i, v in enumerate(h)])


def run(table, fn, keys, lanes):
    import torch

    words, offs = pack(keys)
    out = torch.empty(len(keys), dtype=torch.int32, device="cuda")
    fn(dev(words), dev(offs), len(keys), len(words), out, lanes=lanes)
    decoded = torch.empty((len(keys), 10), dtype=torch.int32, device="cuda")
    table.read(out, len(keys), decoded)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32), decoded.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("lanes", [1, 8])
def test_static_find_or_add_matches_arena_version(svdag_lib, lanes):
    dag = svdag_lib.MyGPUHashDAG(10, pool_bytes=1 << 30)
    arena = dag.create_table(0, [97] * 9)
    static = dag.create_table(0, [97] * 9)
    rng = np.random.default_rng(4242 + lanes)
    base = node_keys(rng, 30000)
    batches = [
        # first call: every key once or twice, shuffled
        [base[i] for i in rng.permutation(np.concatenate([np.arange(30000), np.arange(0, 30000, 2)]))],
        # second call in a row: half already stored, half new, with duplicates
        [k for k in (base[:12000] + node_keys(rng, 18000)) for _ in range(2)],
        # third call: exactly the largest batch, so the probe table fills the whole fixed array
        [k for k in (base[20000:28000] + node_keys(rng, 24768)) for _ in range(2)],
    ]
    assert len(batches[2]) == MAX_KEYS
    for keys in batches:
        assert len(keys) <= MAX_KEYS
        rng.shuffle(keys)
        h_a, w_a = run(arena, arena.find_or_add, keys, lanes)
        h_s, w_s = run(static, static.find_or_add_static, keys, lanes)
        dag.sync()
        for i, k in enumerate(keys):
            assert tuple(w_a[i][: len(k)]) == k
            assert tuple(w_s[i][: len(k)]) == k
        assert np.array_equal(labels(h_a), labels(h_s))  # the same keys share a slot in both tables
        assert arena.stats().items == static.stats().items
    assert static.stats().items == len(set(base) | set(batches[1]) | set(batches[2]))
    dag.free()


def test_static_find_or_add_rejects_oversized_batches(svdag_lib):
    import torch

    dag = svdag_lib.MyGPUHashDAG(10, pool_bytes=1 << 28)
    t = dag.create_table(0, [16] * 9)
    n = MAX_KEYS + 1
    words = np.tile(np.array([1, 7], dtype=np.uint32), n)
    offs = np.arange(0, 2 * n, 2, dtype=np.uint32)
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    with pytest.raises(svdag_lib.SvdagError) as e:
        t.find_or_add_static(dev(words), dev(offs), n, len(words), out)
    assert e.value.status == 1
    dag.free()
