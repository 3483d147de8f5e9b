// Project-written oneTBB stand-in (oracle build only): tbb::parallel_for.
#pragma once
#include "oneapi/tbb/_shim_core.h"
#include "oneapi/tbb/blocked_range.h"

#include <algorithm>
#include <cstddef>

namespace tbb {
inline namespace ktb_v1 {

// Range form: the range is cut into pieces of at most grainsize elements and
// body is called once per piece.
template <typename Value, typename Body>
void parallel_for(const blocked_range<Value> &range, const Body &body) {
    if (range.empty()) return;
    const std::size_t n = range.size();
    const std::size_t g = range.grainsize();
    const std::size_t chunks = (n + g - 1) / g;
    ktb_shim::for_chunks(chunks, [&](std::size_t c) {
        const Value a = static_cast<Value>(range.begin() + c * g);
        const Value b = static_cast<Value>(range.begin() + std::min(n, (c + 1) * g));
        body(blocked_range<Value>(a, b, g));
    });
}

// Index form: f(i) for i in [first, last).
template <typename Index, typename Function>
void parallel_for(Index first, Index last, const Function &f) {
    if (!(first < last)) return;
    const std::size_t n = static_cast<std::size_t>(last - first);
    ktb_shim::for_chunks(n, [&](std::size_t c) { f(static_cast<Index>(first + c)); });
}

}  // namespace ktb_v1
}  // namespace tbb
