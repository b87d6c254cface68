// svdag_snapshot.h - validation of item snapshots (svdag_load_items): splitting a level's words into
// its items and checking each against the level below. Plain C++, so the tests compile the same
// functions for the host.
#pragma once
#include <cstdint>
#include <vector>

#include "svdag_hash.h"

namespace svdag {
namespace snapshot {

// Words of the item starting at p (avail words readable), or 0 when it does not fit or is invalid.
inline uint32_t item_words(bool leaf, const uint32_t* p, uint64_t avail)
{
    if (avail < 2)
        return 0;
    const uint32_t n = leaf ? leaf_words(p[0], p[1]) : node_words(p[0]);
    if (leaf ? (p[0] == 0 && p[1] == 0) : (p[0] & 0xFFu) == 0)
        return 0; // an empty item never occurs in a DAG
    return n <= avail ? n : 0;
}

// Offsets of the items of one level of a snapshot; false when the words do not split into exactly
// `count` items or a child ordinal is out of range.
inline bool split_level(bool leaf, const uint32_t* w, uint64_t nWords, uint64_t count, uint64_t childCount, std::vector<uint64_t>& offs)
{
    offs.clear();
    offs.reserve(count);
    uint64_t at = 0;
    while (at < nWords) {
        const uint32_t n = item_words(leaf, w + at, nWords - at);
        if (!n)
            return false;
        if (!leaf)
            for (uint32_t i = 1; i < n; ++i)
                if (w[at + i] >= childCount)
                    return false;
        offs.push_back(at);
        at += n;
    }
    return offs.size() == count;
}

} // namespace snapshot
} // namespace svdag
