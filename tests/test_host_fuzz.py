"""Host parsers given malformed input: replay text and BasicDAG node arrays of random content must be
rejected with a status (or parsed), never crash the process or read outside the given buffer."""
import ctypes as C

import numpy as np


def test_replay_parser_survives_random_text(svdag_lib):
    L = svdag_lib.lib()
    rng = np.random.default_rng(5)
    alphabet = list(b"EditSphereCubeCopyPaintFillUndoRedoEndFrameSetLocationRotationToolParameters,0123456789.-etruefals\n\r ")
    out = (svdag_lib.ReplayAction * 64)()
    count, bad = C.c_uint64(), C.c_uint64()
    outcomes = set()
    for _ in range(400):
        n = int(rng.integers(0, 300))
        text = bytes(rng.choice(alphabet, n).astype(np.uint8)) if n else b""
        st = L.svdag_replay_parse(text, len(text), 1.0, C.addressof(out), 64, C.byref(count), C.byref(bad))
        assert st in (0, 1, 2)
        outcomes.add(st)
    # well-formed lines around garbage: the parse stops at the bad line and reports it
    text = b"Undo\nEndFrame\nEditSphere,1,2,3\nRedo\n"
    assert L.svdag_replay_parse(text, len(text), 1.0, C.addressof(out), 64, C.byref(count), C.byref(bad)) == 1
    assert bad.value == 2
    assert 1 in outcomes


def test_basic_dag_conversion_survives_random_arrays(svdag_lib):
    L = svdag_lib.lib()
    rng = np.random.default_rng(6)
    lw, li, total = np.zeros(16, np.uint64), np.zeros(16, np.uint64), C.c_uint64()
    for k in range(300):
        levels = int(rng.integers(4, 8))
        n = int(rng.integers(1, 200))
        if k % 3 == 0:  # small values: indices mostly in range, masks with few children
            data = rng.integers(0, n + 4, n).astype(np.uint32)
        else:
            data = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
        cap = 4096
        out = np.zeros(cap, np.uint32)
        st = L.svdag_basic_dag_to_items(data.ctypes.data, n, levels, 1, out.ctypes.data, cap, lw.ctypes.data, li.ctypes.data,
                                        C.byref(total))
        assert st in (0, 2, 4)  # converted, more words than the capacity, or corrupt input
