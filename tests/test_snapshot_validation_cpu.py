"""The item-snapshot validation svdag_load_items runs on the host (svdag_snapshot.h, compiled for the
host by tests/snapshot_host.cpp): every level of snapshots converted from BasicDAGs splits into its
items at the offsets a walk of the item encodings gives, and each kind of malformed level is
rejected: a truncated item, a child ordinal past the level below, an empty node or leaf, a wrong item
count, trailing words."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from test_io import build_basic_dag, random_grid

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def snap(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    so = str(tmp_path_factory.mktemp("snap") / "snapshot_host.so")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", os.path.join(HERE, "snapshot_host.cpp"), "-o", so])
    lib = C.CDLL(so)
    lib.snapshot_split.restype = C.c_int64
    lib.snapshot_split.argtypes = [C.c_int, C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_uint64]
    return lib


def split(snap, leaf, w, count, below):
    w = np.ascontiguousarray(w, dtype=np.uint32)
    offs = np.zeros(max(count, 1) + 8, np.uint64)
    n = snap.snapshot_split(int(leaf), w.ctypes.data, len(w), count, below, offs.ctypes.data, len(offs))
    return None if n < 0 else offs[:n]


def walk(leaf, w):
    """Item offsets by the encodings: node = 1 + popcount(mask byte), leaf = 2 + ceil(4 v / 32)."""
    offs, at = [], 0
    while at < len(w):
        offs.append(at)
        if leaf:
            v = bin(int(w[at])).count("1") + bin(int(w[at + 1])).count("1")
            at += 2 + (4 * v + 31) // 32
        else:
            at += 1 + bin(int(w[at]) & 0xFF).count("1")
    return offs


def levels_of(s):
    out, at = [], 0
    for l in range(s.levels - 1):
        n = int(s.level_words[l])
        out.append(s.words[at:at + n].copy())
        at += n
    return out


@pytest.mark.parametrize("levels,seed", [(5, 0), (6, 1), (7, 2)])
def test_valid_levels_split_like_the_encodings(svdag_lib, snap, levels, seed):
    s = svdag_lib.basic_dag_to_items(build_basic_dag(random_grid(np.random.default_rng(seed), levels), levels), levels, 3)
    lv = levels_of(s)
    LL = levels - 2
    for l, w in enumerate(lv):
        below = int(s.level_items[l + 1]) if l < LL else 0
        got = split(snap, l == LL, w, int(s.level_items[l]), below)
        assert got is not None and list(map(int, got)) == walk(l == LL, w)


@pytest.mark.parametrize("bad", ["truncated", "child_past_below", "empty_node", "empty_leaf", "count_high",
                                 "count_low", "trailing_word"])
def test_malformed_levels_are_rejected(svdag_lib, snap, bad):
    levels = 6
    s = svdag_lib.basic_dag_to_items(build_basic_dag(random_grid(np.random.default_rng(7), levels), levels), levels, 2)
    lv = levels_of(s)
    LL = levels - 2
    l = 2 if bad != "empty_leaf" else LL
    w = lv[l].copy()
    count = int(s.level_items[l])
    below = int(s.level_items[l + 1]) if l < LL else 0
    assert split(snap, l == LL, w, count, below) is not None  # the level as converted is valid
    if bad == "truncated":
        w = w[:-1]
    elif bad == "child_past_below":
        w[1] = below  # the first node's first child ordinal, one past the last item below
    elif bad == "empty_node":
        w[0] = np.uint32(int(w[0]) & 0xFFFFFF00)
    elif bad == "empty_leaf":
        w[0] = w[1] = 0
    elif bad == "count_high":
        count += 1
    elif bad == "count_low":
        count -= 1
    else:
        w = np.concatenate([w, np.array([1, 0], np.uint32)])  # a whole extra node (one child, ordinal 0)
    assert split(snap, l == LL, w, count, below) is None
