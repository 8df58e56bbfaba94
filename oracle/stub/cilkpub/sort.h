// TEST INFRASTRUCTURE ONLY.  Stand-in for Cilkpub's parallel sort, which needs
// a Cilk Plus compiler (absent here): the reference's graph tools sort with
// strict total orders, so any correct sort yields the same sequence.
#pragma once
#include <algorithm>
namespace cilkpub {
template <typename It, typename Cmp>
void cilk_sort(It begin, It end, Cmp cmp) {
  std::sort(begin, end, cmp);
}
template <typename It>
void cilk_sort(It begin, It end) {
  std::sort(begin, end);
}
}  // namespace cilkpub
