"""Item snapshots in tests: building one from the oracle's item export, and comparing two
structurally (canonical ids per level, so item order and handles do not matter)."""
import numpy as np


def leaf_words(lo, hi):
    v = bin(int(lo)).count("1") + bin(int(hi)).count("1")
    return 2 + (v * 4 + 31) // 32


def node_words(header):
    return 1 + bin(int(header) & 0xFF).count("1")


def snapshot_from_rows(svdag, levels, rows):
    """The oracle's export_items rows (10 words, children as row indices, row 0 = the root) as an
    ItemSnapshot: each level's items in first-visit order, children as ordinals."""
    LL = levels - 2
    nl = levels - 1
    lw, li = np.zeros(nl, np.uint64), np.zeros(nl, np.uint64)
    if len(rows) == 0:
        return svdag.ItemSnapshot(levels, np.zeros(0, np.uint32), lw, li)
    words = []
    frontier = [0]
    for level in range(LL + 1):
        order, nxt, out = {}, [], []
        for r in frontier:
            w = rows[r]
            if level == LL:
                out.extend(int(x) for x in w[: leaf_words(w[0], w[1])])
                continue
            n = node_words(w[0])
            out.append(int(w[0]))
            for c in w[1:n]:
                c = int(c)
                if c not in order:
                    order[c] = len(nxt)
                    nxt.append(c)
                out.append(order[c])
        lw[level], li[level] = len(out), len(frontier)
        words.extend(out)
        frontier = nxt
    return svdag.ItemSnapshot(levels, np.array(words, np.uint32), lw, li)


def split(levels, words, level_words):
    at, out = 0, []
    for n in level_words:
        out.append(np.asarray(words[at: at + int(n)]))
        at += int(n)
    return out


def canon(levels, words, level_words, level_items, interner):
    """(root id, per-level sets of ids): each item's id is interned from its level and its words with
    children replaced by their ids, so equal structures get equal ids in one interner."""
    LL = levels - 2
    per = split(levels, words, level_words)
    below, sets = None, [None] * (LL + 1)
    for level in range(LL, -1, -1):
        w, i, ids = per[level], 0, []
        while i < len(w):
            if level == LL:
                n = leaf_words(w[i], w[i + 1])
                key = (level,) + tuple(int(x) for x in w[i: i + n])
            else:
                n = node_words(w[i])
                key = (level, int(w[i])) + tuple(below[int(c)] for c in w[i + 1: i + n])
            ids.append(interner.setdefault(key, len(interner)))
            i += n
        assert len(ids) == int(level_items[level])
        sets[level] = frozenset(ids)
        below = ids
    return (below[0] if below else None), sets


def same_dag(levels, a, b):
    """True when two snapshots (words, level_words, level_items) hold the same DAG."""
    interner = {}
    return canon(levels, *a, interner) == canon(levels, *b, interner)


def snap_parts(snap):
    return snap.words, snap.level_words, snap.level_items
