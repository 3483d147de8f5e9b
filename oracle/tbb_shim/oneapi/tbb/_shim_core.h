// Project-written stand-in for the handful of oneTBB entry points that the
// reference's datamodel/, util/, geometry/, adaptor/ and globalPlacer/simpl/
// sources include. oneTBB itself is an un-checked-out submodule of the
// reference (third_party/oneTBB), so this shim lets those sources compile
// unmodified for the oracle build.
//
// Test infrastructure only: the oracle and the timed CPU baseline link it;
// the CUDA product never does.
//
// Scheduling: when compiled with -fopenmp every construct becomes OpenMP
// tasks (so a parallel_for nested inside a parallel_invoke still spreads over
// all threads); without -fopenmp everything runs serially in index order.
// Work splitting never changes results of the reference code, whose parallel
// bodies write disjoint outputs and whose reductions sum fixed-size chunks in
// a fixed order (globalPlacer/simpl/simpl_parallel.h:35-51).
#pragma once

#include <cstddef>
#include <utility>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace ktb_shim {

// Run f() inside an OpenMP parallel region with a single producer thread, or
// directly when already inside one (a task of an enclosing construct).
template <typename F>
void with_team(F &&f) {
#ifdef _OPENMP
    if (omp_in_parallel()) {
        f();
    } else {
#pragma omp parallel
#pragma omp single
        f();
    }
#else
    f();
#endif
}

// Calls body(c) for every chunk index c in [0, chunks).
template <typename Body>
void for_chunks(std::size_t chunks, const Body &body) {
#ifdef _OPENMP
    if (chunks <= 1) {
        for (std::size_t c = 0; c < chunks; ++c) body(c);
        return;
    }
    with_team([&] {
#pragma omp taskloop grainsize(1)
        for (std::size_t c = 0; c < chunks; ++c) body(c);
    });
#else
    for (std::size_t c = 0; c < chunks; ++c) body(c);
#endif
}

}  // namespace ktb_shim
