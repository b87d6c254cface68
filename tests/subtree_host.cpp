// Host build of the library's subtree-edit geometry (gpu-svdag-editing_b200/csrc/svdag_subtree.h) for
// tests/test_subtree_cpu.py.
#include "../gpu-svdag-editing_b200/csrc/svdag_subtree.h"

extern "C" {
int subtree_node_of(const float* lo, const float* hi, uint32_t levels, uint32_t* level, uint32_t* path)
{
    return svdag::subtree::node_of(lo, hi, levels, *level, path) ? 1 : 0;
}
int subtree_disjoint(uint32_t la, const uint32_t* pa, uint32_t lb, const uint32_t* pb)
{
    return svdag::subtree::disjoint(la, pa, lb, pb) ? 1 : 0;
}
}
