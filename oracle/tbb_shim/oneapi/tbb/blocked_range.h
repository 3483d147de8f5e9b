// Project-written oneTBB stand-in (oracle build only): tbb::blocked_range.
#pragma once
#include <cstddef>

namespace tbb {
inline namespace ktb_v1 {

template <typename Value>
class blocked_range {
public:
    using const_iterator = Value;
    using size_type = std::size_t;

    blocked_range(Value begin, Value end, size_type grainsize = 1)
        : lo(begin), hi(end), grain(grainsize == 0 ? 1 : grainsize) {}

    Value begin() const { return lo; }
    Value end() const { return hi; }
    size_type size() const { return static_cast<size_type>(hi - lo); }
    size_type grainsize() const { return grain; }
    bool empty() const { return !(lo < hi); }
    bool is_divisible() const { return grain < size(); }

private:
    Value lo;
    Value hi;
    size_type grain;
};

}  // namespace ktb_v1
}  // namespace tbb
