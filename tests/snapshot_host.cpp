// Host build of the item-snapshot validation (gpu-svdag-editing_b200/csrc/svdag_snapshot.h) that
// svdag_load_items runs before it touches the GPU. Test infrastructure only.
#include "../gpu-svdag-editing_b200/csrc/svdag_snapshot.h"

extern "C" {

// Items of one level: their count written to offs[0..] (at most cap), or -1 when split_level rejects it.
int64_t snapshot_split(int leaf, const uint32_t* words, uint64_t nWords, uint64_t count, uint64_t childCount,
    uint64_t* offs, uint64_t cap)
{
    std::vector<uint64_t> o;
    if (!svdag::snapshot::split_level(leaf != 0, words, nWords, count, childCount, o))
        return -1;
    for (uint64_t i = 0; i < o.size() && i < cap; ++i)
        offs[i] = o[i];
    return (int64_t)o.size();
}

} // extern "C"
