// Minimal stand-in for TBB's parallel_for_each (TBB is absent from this machine): a sequential
// loop. Only the declarations the reference headers compiled by oracle/build_ref.py include are
// needed; the harness never calls a function that uses it. Test infrastructure only.
#pragma once
#include <algorithm>
#include <iterator>

namespace tbb {
template <class It, class F>
void parallel_for_each(It first, It last, F f) { std::for_each(first, last, f); }
template <class R, class F>
void parallel_for_each(R& range, F f) { std::for_each(std::begin(range), std::end(range), f); }
} // namespace tbb
