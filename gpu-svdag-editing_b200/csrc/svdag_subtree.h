// svdag_subtree.h - the node of a subtree edit: host geometry for grouping the small edits of a batch
// into subtree edits (k_edit_subtrees). Plain C++, so the tests compile the same function for the host.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>

namespace svdag {
namespace subtree {

// The deepest node below the root, at most at level levels - 3 (the level above the leaves), whose
// region holds the footprint box [lo, hi] grown by two voxels; the tools' float tests only ever reach
// nodes that meet the footprint. Returns false when only the root holds it or the box lies off the
// grid. `path` receives the node's coordinates at its level.
inline bool node_of(const float lo[3], const float hi[3], uint32_t levels, uint32_t& level, uint32_t path[3])
{
    const long long size = 1ll << levels;
    long long a[3], b[3];
    for (int k = 0; k < 3; ++k) {
        if (!std::isfinite(lo[k]) || !std::isfinite(hi[k]))
            return false;
        a[k] = (long long)std::floor((double)lo[k]) - 2;
        b[k] = (long long)std::ceil((double)hi[k]) + 2;
        if (b[k] < 0 || a[k] >= size)
            return false;
        a[k] = std::max(a[k], 0ll);
        b[k] = std::min(b[k], size - 1);
    }
    uint32_t L = 0;
    for (uint32_t l = 1; l + 3 <= levels; ++l) {
        const uint32_t sh = levels - l;
        if ((a[0] >> sh) != (b[0] >> sh) || (a[1] >> sh) != (b[1] >> sh) || (a[2] >> sh) != (b[2] >> sh))
            break;
        L = l;
    }
    if (L == 0)
        return false;
    level = L;
    for (int k = 0; k < 3; ++k)
        path[k] = (uint32_t)(a[k] >> (levels - L));
    return true;
}

// Two nodes are disjoint when neither is the other or an ancestor of it.
inline bool disjoint(uint32_t la, const uint32_t* pa, uint32_t lb, const uint32_t* pb)
{
    if (la > lb) {
        std::swap(la, lb);
        std::swap(pa, pb);
    }
    const uint32_t sh = lb - la;
    return (pb[0] >> sh) != pa[0] || (pb[1] >> sh) != pa[1] || (pb[2] >> sh) != pa[2];
}

} // namespace subtree
} // namespace svdag
