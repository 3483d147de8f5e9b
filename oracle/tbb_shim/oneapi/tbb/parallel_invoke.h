// Project-written oneTBB stand-in (oracle build only): tbb::parallel_invoke.
#pragma once
#include "oneapi/tbb/_shim_core.h"

namespace tbb {
inline namespace ktb_v1 {

namespace detail_shim {
template <typename F>
void spawn(const F &f) {
#ifdef _OPENMP
    const F *fp = &f;
#pragma omp task firstprivate(fp)
    (*fp)();
#else
    f();
#endif
}
}  // namespace detail_shim

template <typename... Fs>
void parallel_invoke(const Fs &...fs) {
#ifdef _OPENMP
    ktb_shim::with_team([&] {
        (detail_shim::spawn(fs), ...);
#pragma omp taskwait
    });
#else
    (fs(), ...);
#endif
}

}  // namespace ktb_v1
}  // namespace tbb
