// Project-written oneTBB stand-in (oracle build only): tbb::parallel_sort.
// The reference only sorts with total-order comparators, so std::sort gives
// the same result.
#pragma once
#include <algorithm>

namespace tbb {
inline namespace ktb_v1 {

template <typename It, typename Compare>
void parallel_sort(It first, It last, const Compare &comp) {
    std::sort(first, last, comp);
}

template <typename It>
void parallel_sort(It first, It last) {
    std::sort(first, last);
}

}  // namespace ktb_v1
}  // namespace tbb
