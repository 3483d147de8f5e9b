// Project-written oneTBB stand-in (oracle build only): tbb::parallel_reduce
// (functional form). Pieces are reduced independently and joined in index
// order.
#pragma once
#include "oneapi/tbb/_shim_core.h"
#include "oneapi/tbb/blocked_range.h"

#include <algorithm>
#include <cstddef>
#include <vector>

namespace tbb {
inline namespace ktb_v1 {

template <typename Value, typename T, typename RealBody, typename Reduction>
T parallel_reduce(const blocked_range<Value> &range, const T &identity, const RealBody &body,
                  const Reduction &join) {
    if (range.empty()) return identity;
    const std::size_t n = range.size();
    const std::size_t g = std::max<std::size_t>(range.grainsize(), 1024);
    const std::size_t chunks = (n + g - 1) / g;
    std::vector<T> part(chunks, identity);
    ktb_shim::for_chunks(chunks, [&](std::size_t c) {
        const Value a = static_cast<Value>(range.begin() + c * g);
        const Value b = static_cast<Value>(range.begin() + std::min(n, (c + 1) * g));
        part[c] = body(blocked_range<Value>(a, b, g), identity);
    });
    T acc = identity;
    for (const T &p : part) acc = join(acc, p);
    return acc;
}

}  // namespace ktb_v1
}  // namespace tbb
