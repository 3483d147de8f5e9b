// Warp-tile sparse row sums for the persistent solvers (sm_100a).
//
// Each warp takes 32 consecutive rows of its block and streams their
// (contiguous) nonzeros in chunks of kTileChunk, every lane loading
// consecutive entries: coalesced column and value loads and kTileQ
// independent gathers in flight per lane (FP32 tiles issue the next chunk's
// column loads behind them). The products go to the warp's
// slice of shared memory and each lane adds its own row's products in
// storage order onto the row's first term, carrying the running sum across
// chunks, so every row sum is the same sequence of roundings as a
// row-per-thread loop (and, in FP64, as the reference's
// SparseSystem::multiply, simpl_lss.h:49-57). Where a lane's run of
// products is 16-byte aligned it reads two per shared load.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ktg {

constexpr int kTileQ = 4;
constexpr int kTileChunk = 32 * kTileQ;

template <typename T>
struct TilePair;
template <>
struct TilePair<double> {
    using type = double2;
};
template <>
struct TilePair<float> {
    using type = float2;
};

// Work per row when the block's rows are split between its warps: the row's
// nonzeros plus this many (row pointers, the row's own terms, the emit);
// 2 measured best of {2, 8, 24} on the 211k and 1M systems.
constexpr int32_t kRowCost = 2;

// Contiguous row ranges of the block's warps, balanced by kRowCost plus the
// nonzeros of each row: warp w takes rows [wb[w], wb[w+1]) of [0, R).
// cost(l) is the (nondecreasing) work of rows [0, l). Every row sum stays
// the same; only which lane adds it changes, and that depends on the matrix
// pattern alone, so results are still the same from run to run. All threads
// of the block call it; wb has room for the warp count + 1.
template <class Cost>
__device__ __forceinline__ void warp_row_bounds(int32_t R, int32_t *wb, Cost cost) {
    const int nw = blockDim.x >> 5;
    const int w = threadIdx.x;
    if (w <= nw) {
        int32_t res = w == 0 ? 0 : R;
        if (w > 0 && w < nw) {
            const int64_t target = cost(R) * w / nw;
            int32_t lo = 0, hi = R;  // smallest l with cost(l) >= target
            while (lo < hi) {
                const int32_t mid = lo + (hi - lo) / 2;
                if (cost(mid) >= target)
                    hi = mid;
                else
                    lo = mid + 1;
            }
            res = lo;
        }
        wb[w] = res;
    }
    __syncthreads();
}

// Per-axis flags as a bit mask (bit a: axis a), passed by value so that a
// kernel's flags stay in registers (a bool array indexed by a runtime axis
// would live in local memory).
constexpr unsigned kAllAxes = 3u;
__device__ __forceinline__ unsigned axis_mask(bool a0, bool a1) {
    return (a0 ? 1u : 0u) | (a1 ? 2u : 0u);
}

// Rows [r0, r0 + R) of a block's slice of the combined row space
// [axis 0 rows | axis 1 rows] (axis 1 starts at row n0); rows of an axis
// whose bit in `live` is clear are skipped. All threads of the block call
// it.
//   wb: per-warp row ranges from warp_row_bounds, or null for tiles dealt
//       to the warps in turn (warp w takes tiles w, w + nw, ...);
//   csr(pass, rp, col, val, in): the axis's CSR arrays and gathered vector;
//   start(l, pass, i) -> T: the row's first term (diag * own value);
//   emit(l, pass, i, sum): the finished row sum.
// tilebuf holds kTileChunk elements per warp, 16-byte aligned.
template <typename T, class Csr, class Start, class Emit>
__device__ __forceinline__ void warp_tile_spmv(int32_t r0, int32_t n0, int32_t R, unsigned live,
                                               const int32_t *wb, T *tilebuf, Csr csr, Start start,
                                               Emit emit) {
    using P2 = typename TilePair<T>::type;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    T *buf = tilebuf + warp * kTileChunk;
    const int32_t first = wb ? wb[warp] : warp * 32;
    const int32_t end = wb ? wb[warp + 1] : R;
    const int32_t step = wb ? 32 : nw * 32;
    for (int32_t t0 = first; t0 < end; t0 += step) {
        const int32_t l = t0 + lane;
        const int32_t c = r0 + l;
        const int axis = c >= n0 ? 1 : 0;
        const int32_t i = c - (axis ? n0 : 0);
        const bool mine = l < end && ((live >> axis) & 1u);
        // a tile that straddles the axis boundary takes one pass per axis
#pragma unroll 1
        for (int pass = 0; pass < 2; ++pass) {
            const bool part = mine && axis == pass;
            const unsigned m = __ballot_sync(0xffffffffu, part);
            if (!m) continue;
            const int32_t *rp, *col;
            const T *val, *in;
            csr(pass, rp, col, val, in);
            int32_t rs = 0, re = 0;
            T sum = T(0);
            if (part) {
                rs = __ldg(rp + i);
                re = __ldg(rp + i + 1);
                sum = start(l, pass, i);
            }
            // the participating rows are consecutive: their entries are
            // [rs of the first, re of the last)
            const int32_t k_begin = __shfl_sync(0xffffffffu, rs, __ffs(m) - 1);
            const int32_t k_end = __shfl_sync(0xffffffffu, re, 31 - __clz(m));
            int32_t cl[kTileQ];
            auto load_cols = [&](int32_t kb) {
#pragma unroll
                for (int q = 0; q < kTileQ; ++q) {
                    const int32_t k = kb + lane + 32 * q;
                    cl[q] = k < k_end ? __ldg(col + k) : -1;
                }
            };
            // FP32 tiles load the next chunk's columns while the chunk's own
            // gathers are in flight (one memory round trip per chunk instead
            // of two; 3% off the FP32 solves at 211k cells). The FP64 tiles
            // keep the plain order: with their 8-byte products the extra
            // registers cost the register-capped FP64 solve about as much.
            constexpr bool kAhead = sizeof(T) == 4;
            if (kAhead) load_cols(k_begin);
#pragma unroll 1
            for (int32_t k0 = k_begin; k0 < k_end; k0 += kTileChunk) {
                if (!kAhead) load_cols(k0);
                T pr[kTileQ];
#pragma unroll
                for (int q = 0; q < kTileQ; ++q) {
                    const int32_t k = k0 + lane + 32 * q;
                    pr[q] = cl[q] >= 0 ? __ldg(val + k) * __ldcg(in + cl[q]) : T(0);
                }
                if (kAhead) load_cols(k0 + kTileChunk);
#pragma unroll
                for (int q = 0; q < kTileQ; ++q) buf[lane + 32 * q] = pr[q];
                __syncwarp();
                if (part) {
                    int32_t j = (rs > k0 ? rs : k0) - k0;
                    const int32_t je = (re < k0 + kTileChunk ? re : k0 + kTileChunk) - k0;
                    if ((j & 1) && j < je) sum += buf[j++];
                    for (; j + 1 < je; j += 2) {
                        const P2 t = *reinterpret_cast<const P2 *>(buf + j);
                        sum += t.x;
                        sum += t.y;
                    }
                    if (j < je) sum += buf[j];
                }
                __syncwarp();
            }
            if (part) emit(l, pass, i, sum);
        }
    }
}

}  // namespace ktg
