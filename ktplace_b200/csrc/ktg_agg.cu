// Aggregation (block-Jacobi) preconditioner for the mixed-precision solve.
//
// B2B systems are dominated by a few very strong couplings (two pins of a net
// a floor-distance apart get weight base / floor), which point Jacobi cannot
// see. Three levels of pairwise aggregation by strength group the rows into
// aggregates of at most 8 rows; the preconditioner is the exact inverse of
// A's diagonal block on every aggregate. The rows are renumbered so that
// each aggregate is contiguous and the mixed PCG never splits one between
// two thread blocks: applying M is then a small dense product from the
// block's own shared-memory slice (no gather, no extra grid barrier).
//
// The x and y systems are handled as one block-diagonal system of 2n rows
// (row c < n is x row c, c >= n is y row c - n). Everything is
// deterministic: matching by handshake on strengths with index tie-breaks,
// Galerkin sums in raw storage order, numbering by prefix sums.
//
// Level rules (one level = matching + coarsening):
//   strength of a stored entry (I, J, v): s = -v / sqrt(d_I d_J)
//   kRounds handshake rounds: each unmatched I picks the unmatched J != I of
//     largest s > 0 (ties: smaller J); mutual picks are matched;
//   leaders (unmatched, or the smaller of a pair) are numbered in order;
//   coarse row of J = (a, b): entries of row a then row b mapped to coarse
//     ids, those landing on J summed into the coarse diagonal, the others
//     summed per id in that raw order and stored with the ids ascending.
//
// Device memory (per context, grown with the systems): level arrays over 2n
// nodes (mate, pick, flags, ids, children, sizes), two compact coarse CSRs
// of nnz(x) + nnz(y) entries, and the permuted system (row_ptr, col, FP64 and
// FP32 values, diag, rhs, x) plus the block inverses (8 floats per row).
#include "ktg_agg.h"
#include "ktg_coarse_head.cuh"
#include "ktg_common.cuh"
#include "ktg_context.h"
#include "ktg_spmv.cuh"

#include <algorithm>

namespace ktg {

namespace {

constexpr int kRounds = 2;
constexpr int kLevels = 3;
constexpr int kAggMax = 8;
constexpr int kT = 256;
constexpr int kScanTile = 2048;  // 1024 threads x 2

// Rows of one level: the two axis CSRs (level 0) or a compact coarse CSR.
// Axis arrays are separate fields chosen with a conditional, so that no
// thread copies the parameter block to local memory.
struct LevelView {
    bool fine;
    int32_t n;  // rows per axis (level 0)
    const int32_t *rp0, *rp1;
    const int32_t *col0, *col1;
    const double *val0, *val1;
    const double *diag0, *diag1;
    const int32_t *start;
    const int32_t *len;
    const int32_t *ccol;
    const double *cval;
    const double *cdiag;
};

struct RowRef {
    int32_t e0, e1, off;
    const int32_t *col;
    const double *val;
};

__device__ __forceinline__ RowRef row_of(const LevelView &L, int32_t I) {
    RowRef r;
    if (L.fine) {
        const bool y = I >= L.n;
        const int32_t i = y ? I - L.n : I;
        const int32_t *rp = y ? L.rp1 : L.rp0;
        r.e0 = __ldg(rp + i);
        r.e1 = __ldg(rp + i + 1);
        r.off = y ? L.n : 0;
        r.col = y ? L.col1 : L.col0;
        r.val = y ? L.val1 : L.val0;
    } else {
        r.e0 = __ldg(L.start + I);
        r.e1 = r.e0 + __ldg(L.len + I);
        r.off = 0;
        r.col = L.ccol;
        r.val = L.cval;
    }
    return r;
}

__device__ __forceinline__ double diag_of(const LevelView &L, int32_t I) {
    if (L.fine) {
        const bool y = I >= L.n;
        return __ldg((y ? L.diag1 : L.diag0) + (y ? I - L.n : I));
    }
    return __ldg(L.cdiag + I);
}

__global__ void k_init(int32_t rows, int32_t *cur, int32_t *pos, int32_t *size, int32_t *mate,
                       int32_t *counts) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) {
        for (int k = 0; k < 8; ++k) counts[k] = 0;
        counts[0] = rows;
        counts[6] = rows;
    }
    if (c >= rows) return;
    cur[c] = c;
    pos[c] = 0;
    size[c] = 1;
    mate[c] = -1;
}

// One warp per 32 consecutive nodes (CSR-vector form): the lanes walk the
// flattened entries of the warp's unmatched rows 32 at a time, so every
// lane's gathers (mate and diag of the neighbour) are in flight together
// whatever the row lengths; a segmented shuffle reduction gives each row's
// best entry in the chunk, merged into a per-row slot in shared memory. The
// result (largest strength, ties to the smaller J) is order-free.
constexpr int kPickWarps = 8;

__device__ __forceinline__ void pick_merge(double ob, int32_t oj, double &best, int32_t &bj) {
    if (oj >= 0 && (bj < 0 || ob > best || (ob == best && oj < bj))) {
        best = ob;
        bj = oj;
    }
}

// kFirst (first round of a level: nothing is matched yet): computes every
// entry's strength and stores it in sbuf (y rows of level 0 at offset yoff);
// later rounds read it back and gather only the neighbour's mate.
template <bool kFirst>
__global__ void __launch_bounds__(32 * kPickWarps) k_pick(LevelView L, const int32_t *count,
                                                          const int32_t *mate, int32_t *pick,
                                                          double *sbuf, int64_t yoff) {
    __shared__ double best_s[kPickWarps][32];
    __shared__ int32_t best_j[kPickWarps][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int32_t cnt = *count;
    const int32_t base = (blockIdx.x * kPickWarps + w) * 32;
    if (base >= cnt) return;  // whole warp
    const int32_t I = base + lane;
    bool act = false, yax = false;
    int32_t e0 = 0, len = 0;
    double dI = 1.0;
    if (I < cnt && (kFirst || mate[I] < 0)) {
        act = true;
        const RowRef r = row_of(L, I);
        e0 = r.e0;
        len = r.e1 - r.e0;
        yax = r.off != 0;
        if (kFirst) dI = diag_of(L, I);
    }
    int32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    const int32_t excl = incl - len;
    const int32_t T = __shfl_sync(0xffffffffu, incl, 31);
    best_s[w][lane] = 0.0;
    best_j[w][lane] = -1;
    __syncwarp();
    for (int32_t t0 = 0; t0 < T; t0 += 32) {
        const int32_t t = t0 + lane;
        // row of entry t: the last lane whose exclusive offset is <= t
        int row = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
            const int cand = row + step;
            const int32_t ex = __shfl_sync(0xffffffffu, excl, cand & 31);
            if (cand < 32 && ex <= t) row = cand;
        }
        const int32_t re0 = __shfl_sync(0xffffffffu, e0, row);
        const int32_t rex = __shfl_sync(0xffffffffu, excl, row);
        const bool ry = __shfl_sync(0xffffffffu, yax, row);
        const double rd = __shfl_sync(0xffffffffu, dI, row);
        double sv = 0.0;
        int32_t sj = -1;
        if (t < T) {
            const int32_t e = re0 + (t - rex);
            const int32_t *col = L.fine ? (ry ? L.col1 : L.col0) : L.ccol;
            const int32_t J = __ldg(col + e) + (ry ? L.n : 0);
            double *sp = sbuf + (ry ? yoff : 0) + e;
            double st;
            if (kFirst) {
                const double *val = L.fine ? (ry ? L.val1 : L.val0) : L.cval;
                st = -__ldg(val + e) / sqrt(rd * diag_of(L, J));
                *sp = st;
            } else {
                st = *sp;
            }
            if (J != base + row && st > 0.0 && (kFirst || mate[J] < 0)) {
                sv = st;
                sj = J;
            }
        }
        // segmented max over lanes of the same row (contiguous in the chunk)
        const int rowv = t < T ? row : -1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double os = __shfl_down_sync(0xffffffffu, sv, o);
            const int32_t oj = __shfl_down_sync(0xffffffffu, sj, o);
            const int orow = __shfl_down_sync(0xffffffffu, rowv, o);
            if (lane + o < 32 && orow == rowv) pick_merge(os, oj, sv, sj);
        }
        const int prow = __shfl_up_sync(0xffffffffu, rowv, 1);
        if (rowv >= 0 && (lane == 0 || prow != rowv)) {
            double b = best_s[w][rowv];
            int32_t bj = best_j[w][rowv];
            pick_merge(sv, sj, b, bj);
            best_s[w][rowv] = b;
            best_j[w][rowv] = bj;
        }
        __syncwarp();
    }
    if (I < cnt) pick[I] = act ? best_j[w][lane] : -1;
}

__global__ void k_handshake(const int32_t *count, const int32_t *pick, int32_t *mate) {
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= *count) return;
    const int32_t J = pick[I];
    if (mate[I] < 0 && J >= 0 && pick[J] == I) mate[I] = J;
}

__global__ void k_leader_flag(const int32_t *count, const int32_t *mate, int32_t *flag) {
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= *count) return;
    const int32_t m = mate[I];
    flag[I] = (m < 0 || I < m) ? 1 : 0;
}

// ---- exclusive scan of int32 counts (count read on the device) -------------

__device__ __forceinline__ int32_t block_excl_scan(int32_t v, int32_t *warp_tot, int32_t &total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        const int32_t x = lane < nw ? warp_tot[lane] : 0;
        int32_t xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t t = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += t;
        }
        if (lane < nw) warp_tot[lane] = xi - x;
        if (lane == 31) warp_tot[32] = xi;
    }
    __syncthreads();
    total = warp_tot[32];
    const int32_t out = warp_tot[w] + incl - v;
    __syncthreads();
    return out;
}

__global__ void __launch_bounds__(1024) k_scan_tiles(const int32_t *in, int32_t *out,
                                                     const int32_t *count, int32_t *tile_sum) {
    __shared__ int32_t warp_tot[33];
    const int32_t n = *count;
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile;
    if (base >= n && blockIdx.x > 0) return;
    const int64_t i0 = base + 2 * threadIdx.x;
    const int32_t a = i0 < n ? in[i0] : 0;
    const int32_t b = i0 + 1 < n ? in[i0 + 1] : 0;
    int32_t total;
    const int32_t ex = block_excl_scan(a + b, warp_tot, total);
    if (i0 < n) out[i0] = ex;
    if (i0 + 1 < n) out[i0 + 1] = ex + a;
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_sums(int32_t *tile_sum, const int32_t *count,
                                                    int32_t *total_out) {
    __shared__ int32_t warp_tot[33];
    __shared__ int32_t carry;
    const int32_t n = *count;
    const int32_t tiles = n > 0 ? (n + kScanTile - 1) / kScanTile : 0;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int32_t t0 = 0; t0 < tiles; t0 += blockDim.x) {
        const int32_t t = t0 + threadIdx.x;
        const int32_t v = t < tiles ? tile_sum[t] : 0;
        int32_t tot;
        const int32_t ex = block_excl_scan(v, warp_tot, tot);
        if (t < tiles) tile_sum[t] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_add(int32_t *out, const int32_t *count, const int32_t *tile_sum) {
    const int32_t n = *count;
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] += tile_sum[i / kScanTile];
}

// ---- level bookkeeping --------------------------------------------------------

__global__ void k_number(const int32_t *count, const int32_t *mate, const int32_t *scan,
                         int32_t *cid, int32_t *child0, int32_t *child1,
                         const int32_t *size_old, int32_t *size_new) {
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= *count) return;
    const int32_t m = mate[I];
    if (m < 0 || I < m) {
        const int32_t J = scan[I];
        cid[I] = J;
        child0[J] = I;
        child1[J] = m;
        size_new[J] = size_old[I] + (m >= 0 ? size_old[m] : 0);
    } else {
        cid[I] = scan[m];
    }
}

__global__ void k_follow(int32_t rows, int32_t *cur, int32_t *pos, const int32_t *mate,
                         const int32_t *cid, const int32_t *size_old) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= rows) return;
    const int32_t a = cur[c];
    const int32_t m = mate[a];
    if (m >= 0 && m < a) pos[c] += size_old[m];
    cur[c] = cid[a];
}

__global__ void k_reset_mate(const int32_t *count, int32_t *mate) {
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I < *count) mate[I] = -1;
}

// Raw length of every coarse row, and where its children's rows start
// (row a at ea[J] with la[J] entries, row b at eb[J]), so that the coarse
// kernels fetch all of a row's metadata in one round of independent loads.
__global__ void k_rawlen(LevelView L, const int32_t *count, const int32_t *child0,
                         const int32_t *child1, int32_t *rawlen, int32_t *ea, int32_t *eb,
                         int32_t *la_out) {
    const int32_t J = blockIdx.x * blockDim.x + threadIdx.x;
    if (J >= *count) return;
    const RowRef ra = row_of(L, child0[J]);
    const int32_t la = ra.e1 - ra.e0;
    int32_t len = la, e0b = ra.e0;
    const int32_t b = child1[J];
    if (b >= 0) {
        const RowRef rb = row_of(L, b);
        len += rb.e1 - rb.e0;
        e0b = rb.e0;
    }
    rawlen[J] = len;
    ea[J] = ra.e0;
    eb[J] = e0b;
    la_out[J] = la;
}

// Coarse row J = (a, b): the raw entries (row a's, then row b's) mapped to
// coarse ids; ids equal to J fold into the diagonal in raw order
// (d_a, a's entries, d_b, b's entries); the others are summed per id in raw
// order and stored with the ids ascending. Two persistent grid-stride kernels:
//   k_coarse_warp: one warp per row of raw length R <= kWarpRaw, two raw
//     entries per lane in registers; for every entry the warp walks all R
//     entries by shuffles to find whether it is the first of its id, its
//     rank among the distinct ids and its raw-order sum; longer rows are
//     appended to a list (order free: each row is processed on its own);
//   k_coarse_heavy: one block per listed row: bitonic sort of (id, raw
//     index) in shared memory for R <= kHeavyMax, output ranks by a block
//     scan; longer rows by sorted insertion in one thread directly in the
//     output row (rare: rows that long need nets of hundreds of pins).
constexpr int kWarpRaw = 64;
constexpr int kWarpWarps = 8;
constexpr int kHeavyMax = 2048;
constexpr int kHeavyThreads = 256;

struct CoarseArgs {
    LevelView L;
    const int32_t *count;
    const int32_t *child0, *child1, *cid, *start, *rawlen;
    const int32_t *ea, *eb, *la;  // children's row starts and row a's length
    int32_t *out_len, *out_col;
    double *out_val, *out_diag;
    int32_t *heavy;        // rows with R > kWarpRaw
    int32_t *heavy_count;  // zero before k_coarse_warp
};

// Sorted insertion of (K, v) into keys/sums[0..k) (stride apart).
template <typename KeyPtr, typename SumPtr>
__device__ __forceinline__ void sorted_add(KeyPtr keys, SumPtr sums, int stride, int &k,
                                           int32_t K, double v) {
    int p = 0;
    while (p < k && keys[p * stride] < K) ++p;
    if (p < k && keys[p * stride] == K) {
        sums[p * stride] += v;
        return;
    }
    for (int q = k; q > p; --q) {
        keys[q * stride] = keys[(q - 1) * stride];
        sums[q * stride] = sums[(q - 1) * stride];
    }
    keys[p * stride] = K;
    sums[p * stride] = v;
    ++k;
}

// Row references of coarse row J's children from the precomputed starts
// (both children are rows of the same axis at level 0).
__device__ __forceinline__ void child_rows(const CoarseArgs &A, int32_t J, int32_t a, RowRef &ra,
                                           RowRef &rb, int &la) {
    const LevelView &L = A.L;
    la = A.la[J];
    const bool y = L.fine && a >= L.n;
    ra.e0 = A.ea[J];
    ra.e1 = ra.e0 + la;
    ra.off = y ? L.n : 0;
    ra.col = L.fine ? (y ? L.col1 : L.col0) : L.ccol;
    ra.val = L.fine ? (y ? L.val1 : L.val0) : L.cval;
    rb = ra;
    rb.e0 = A.eb[J];
    rb.e1 = rb.e0;  // unused: raw index e >= la selects row b
}

// Raw entry e of coarse row (a, b): its coarse id and value.
__device__ __forceinline__ void raw_entry(const CoarseArgs &A, const RowRef &ra, const RowRef &rb,
                                          int la, int e, int32_t &K, double &v) {
    const bool in_a = e < la;
    const int32_t idx = in_a ? ra.e0 + e : rb.e0 + (e - la);
    K = A.cid[__ldg((in_a ? ra.col : rb.col) + idx) + (in_a ? ra.off : rb.off)];
    v = __ldg((in_a ? ra.val : rb.val) + idx);
}

// Compare-exchange of a bitonic network: keep the smaller key when this
// position should hold the smaller one.
template <typename KeyT>
__device__ __forceinline__ KeyT bitonic_keep(KeyT mine, KeyT other, bool keep_small) {
    const bool less = mine < other;
    return (less == keep_small) ? mine : other;
}

// Bitonic sort of P keys held two per lane (positions 2 * lane and
// 2 * lane + 1), ascending; fully unrolled so every direction mask is a
// constant. Positions at or beyond P (lanes >= P / 2) are left alone.
template <int P, typename KeyT>
__device__ __forceinline__ void bitonic_pairs(KeyT &k0, KeyT &k1, int lane) {
#pragma unroll
    for (int kk = 2; kk <= P; kk <<= 1) {
#pragma unroll
        for (int j = kk >> 1; j > 0; j >>= 1) {
            const int p0 = 2 * lane;
            const bool asc = (p0 & kk) == 0;  // the same for p0 and p0 + 1
            if (j == 1) {
                const KeyT lo = k0 < k1 ? k0 : k1, hi = k0 < k1 ? k1 : k0;
                k0 = asc ? lo : hi;
                k1 = asc ? hi : lo;
            } else {
                const KeyT o0 = __shfl_xor_sync(0xffffffffu, k0, j >> 1);
                const KeyT o1 = __shfl_xor_sync(0xffffffffu, k1, j >> 1);
                const bool keep_small = ((p0 & j) == 0) == asc;  // p0 + 1 has the same bit j
                k0 = bitonic_keep(k0, o0, keep_small);
                k1 = bitonic_keep(k1, o1, keep_small);
            }
        }
    }
}

// Keys are (coarse id << kShift) | raw index: 32-bit when the ids fit in
// 26 bits, else 64-bit.
template <typename KeyT>
__global__ void __launch_bounds__(32 * kWarpWarps) k_coarse_warp(CoarseArgs A) {
    constexpr int kShift = sizeof(KeyT) == 8 ? 32 : 6;
    constexpr KeyT kPad = ~KeyT(0);
    // per warp: the sorted (key, value) sequence, for the segment folds
    __shared__ KeyT skey_s[kWarpWarps][kWarpRaw];
    __shared__ double sval_s[kWarpWarps][kWarpRaw];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    KeyT *skey = skey_s[w];
    double *sval = sval_s[w];
    const LevelView &L = A.L;
    const int32_t cnt = *A.count;
    const int32_t warps = gridDim.x * kWarpWarps;
    for (int32_t J = blockIdx.x * kWarpWarps + w; J < cnt; J += warps) {
        const int32_t R = A.rawlen[J];
        if (R > kWarpRaw) {
            if (lane == 0) A.heavy[atomicAdd(A.heavy_count, 1)] = J;
            continue;
        }
        const int32_t a = A.child0[J], b = A.child1[J];
        RowRef ra, rb;
        int la;
        child_rows(A, J, a, ra, rb, la);
        // positions p = 2 * lane + r hold raw entries e = p (r = 0, 1)
        KeyT k0 = kPad, k1 = kPad;
        double v0 = 0.0, v1 = 0.0;
        {
            const int e0 = 2 * lane, e1 = 2 * lane + 1;
            int32_t K;
            if (e0 < R) {
                raw_entry(A, ra, rb, la, e0, K, v0);
                k0 = (static_cast<KeyT>(static_cast<uint32_t>(K)) << kShift) | KeyT(e0);
            }
            if (e1 < R) {
                raw_entry(A, ra, rb, la, e1, K, v1);
                k1 = (static_cast<KeyT>(static_cast<uint32_t>(K)) << kShift) | KeyT(e1);
            }
        }
        // raw values by raw index, for the folds after the sort
        sval[2 * lane] = v0;
        sval[2 * lane + 1] = v1;
        // bitonic sort of the keys over P = 32 or 64 positions
        if (R <= 32) bitonic_pairs<32>(k0, k1, lane);
        else bitonic_pairs<64>(k0, k1, lane);
        skey[2 * lane] = k0;
        skey[2 * lane + 1] = k1;
        __syncwarp();
        // segment heads: first position of each id; ids != J are output rows
        const uint32_t uJ = static_cast<uint32_t>(J);
        const uint32_t K0 = static_cast<uint32_t>(k0 >> kShift), K1 = static_cast<uint32_t>(k1 >> kShift);
        const uint32_t Kprev = lane == 0 ? 0xffffffffu
                                         : static_cast<uint32_t>(skey[2 * lane - 1] >> kShift);
        const bool in0 = 2 * lane < R, in1 = 2 * lane + 1 < R;
        const bool first0 = in0 && (lane == 0 || Kprev != K0);
        const bool first1 = in1 && K1 != K0;
        const bool h0 = first0 && K0 != uJ, h1 = first1 && K1 != uJ;
        const unsigned b0 = __ballot_sync(0xffffffffu, h0), b1 = __ballot_sync(0xffffffffu, h1);
        const unsigned below = (1u << lane) - 1u;
        const int rank0 = __popc(b0 & below) + __popc(b1 & below);
        const int rank1 = rank0 + (h0 ? 1 : 0);
        const int32_t st = A.start[J];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const bool h = r == 0 ? h0 : h1;
            const bool dh = (r == 0 ? first0 : first1) && (r == 0 ? K0 : K1) == uJ;
            const int p = 2 * lane + r;
            const uint32_t K = r == 0 ? K0 : K1;
            if (h) {
                double sum = sval[static_cast<uint32_t>(skey[p] & ((KeyT(1) << kShift) - 1))];
                for (int q = p + 1; q < R && static_cast<uint32_t>(skey[q] >> kShift) == K; ++q)
                    sum += sval[static_cast<uint32_t>(skey[q] & ((KeyT(1) << kShift) - 1))];
                const int rank = r == 0 ? rank0 : rank1;
                A.out_col[st + rank] = static_cast<int32_t>(K);
                A.out_val[st + rank] = sum;
            }
            if (dh) {
                double dacc = diag_of(L, a);
                bool added_b = false;
                for (int q = p; q < R && static_cast<uint32_t>(skey[q] >> kShift) == K; ++q) {
                    const uint32_t idx = static_cast<uint32_t>(skey[q] & ((KeyT(1) << kShift) - 1));
                    if (!added_b && static_cast<int>(idx) >= la) {
                        dacc += diag_of(L, b);
                        added_b = true;
                    }
                    dacc += sval[idx];
                }
                if (!added_b && b >= 0) dacc += diag_of(L, b);
                A.out_diag[J] = dacc;
            }
        }
        const bool any_diag = __any_sync(0xffffffffu, (first0 && K0 == uJ) || (first1 && K1 == uJ));
        if (lane == 0) {
            A.out_len[J] = __popc(b0) + __popc(b1);
            if (!any_diag) A.out_diag[J] = b >= 0 ? diag_of(L, a) + diag_of(L, b) : diag_of(L, a);
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(kHeavyThreads) k_coarse_heavy(CoarseArgs A) {
    __shared__ unsigned long long key[kHeavyMax];
    __shared__ double vr[kHeavyMax];
    __shared__ int32_t warp_tot[33];
    const LevelView &L = A.L;
    const int tid = threadIdx.x;
    const int32_t nh = *A.heavy_count;
    for (int32_t h = blockIdx.x; h < nh; h += gridDim.x) {
        const int32_t J = A.heavy[h];
        const int32_t R = A.rawlen[J];
        const int32_t a = A.child0[J], b = A.child1[J];
        RowRef ra, rb;
        int la;
        child_rows(A, J, a, ra, rb, la);
        if (R > kHeavyMax) {
            if (tid == 0) {
                int32_t *keys = A.out_col + A.start[J];
                double *sums = A.out_val + A.start[J];
                int k = 0;
                double dacc = diag_of(L, a);
                for (int e = 0; e < R; ++e) {
                    if (e == la) dacc += diag_of(L, b);
                    int32_t K;
                    double v;
                    raw_entry(A, ra, rb, la, e, K, v);
                    if (K == J) dacc += v;
                    else sorted_add(keys, sums, 1, k, K, v);
                }
                if (la == R && b >= 0) dacc += diag_of(L, b);
                A.out_len[J] = k;
                A.out_diag[J] = dacc;
            }
            __syncthreads();
            continue;
        }
        int P = 1;
        while (P < R) P <<= 1;
        for (int e = tid; e < P; e += kHeavyThreads) {
            if (e < R) {
                int32_t K;
                double v;
                raw_entry(A, ra, rb, la, e, K, v);
                key[e] = (static_cast<unsigned long long>(static_cast<uint32_t>(K)) << 32) |
                         static_cast<uint32_t>(e);
                vr[e] = v;
            } else {
                key[e] = ~0ull;
            }
        }
        __syncthreads();
        for (int kk = 2; kk <= P; kk <<= 1) {
            for (int j = kk >> 1; j > 0; j >>= 1) {
                for (int i = tid; i < P; i += kHeavyThreads) {
                    const int ixj = i ^ j;
                    if (ixj > i) {
                        const unsigned long long x = key[i], y = key[ixj];
                        if ((x > y) == ((i & kk) == 0)) {
                            key[i] = y;
                            key[ixj] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
        // segment heads (ids != J) in ascending order, ranked by a block scan
        const uint32_t uJ = static_cast<uint32_t>(J);
        int32_t running = 0;
        int any_diag = 0;
        for (int i0 = 0; i0 < R; i0 += kHeavyThreads) {
            const int i = i0 + tid;
            bool head = false, dhead = false;
            uint32_t K = 0;
            if (i < R) {
                K = static_cast<uint32_t>(key[i] >> 32);
                const bool first = i == 0 || static_cast<uint32_t>(key[i - 1] >> 32) != K;
                head = first && K != uJ;
                dhead = first && K == uJ;
            }
            int32_t tot;
            const int32_t ex = block_excl_scan(head ? 1 : 0, warp_tot, tot);
            if (head) {
                double sum = vr[static_cast<uint32_t>(key[i])];
                for (int q = i + 1; q < R && static_cast<uint32_t>(key[q] >> 32) == K; ++q)
                    sum += vr[static_cast<uint32_t>(key[q])];
                A.out_col[A.start[J] + running + ex] = static_cast<int32_t>(K);
                A.out_val[A.start[J] + running + ex] = sum;
            }
            if (dhead) {
                double dacc = diag_of(L, a);
                bool added_b = false;
                for (int q = i; q < R && static_cast<uint32_t>(key[q] >> 32) == K; ++q) {
                    const uint32_t idx = static_cast<uint32_t>(key[q]);
                    if (!added_b && static_cast<int>(idx) >= la) {
                        dacc += diag_of(L, b);
                        added_b = true;
                    }
                    dacc += vr[idx];
                }
                if (!added_b && b >= 0) dacc += diag_of(L, b);
                A.out_diag[J] = dacc;
            }
            any_diag |= __syncthreads_or(dhead ? 1 : 0);
            running += tot;
        }
        if (tid == 0) {
            A.out_len[J] = running;
            if (!any_diag) A.out_diag[J] = b >= 0 ? diag_of(L, a) + diag_of(L, b) : diag_of(L, a);
        }
        __syncthreads();
    }
}

// ---- final layout, permuted system, block inverses -------------------------

__global__ void k_newpos(int32_t rows, const int32_t *cur, const int32_t *pos,
                         const int32_t *agg_start, int32_t *newpos, int32_t *order) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= rows) return;
    const int32_t p = agg_start[cur[c]] + pos[c];
    newpos[c] = p;
    order[p] = c;
}

__global__ void k_plen(LevelView L, int32_t rows, const int32_t *order, int32_t *plen) {
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= rows) return;
    const RowRef r = row_of(L, order[k]);
    plen[k] = r.e1 - r.e0;
}

// The permuted system as warp tiles: a warp takes 32 consecutive permuted
// rows, whose entries are consecutive in the output; the lanes walk those
// entries 32 at a time (each lane finding its row by a search over the
// warp's exclusive row offsets), so the writes are coalesced and the reads
// stream each source row. Columns renumbered (per-axis local), values in FP64
// and FP32; diag, rhs and the coarse vector's z by the row's own lane (z of
// mode 2 sums the row's |a_ij| in storage order).
constexpr int kPfWarps = 8;
__global__ void __launch_bounds__(32 * kPfWarps)
    k_pfill_tiles(LevelView L, int32_t rows, const int32_t *__restrict__ order,
                  const int32_t *__restrict__ newpos, const int32_t *__restrict__ prp,
                  const double *__restrict__ rhs0, const double *__restrict__ rhs1,
                  int32_t *__restrict__ pcol, double *__restrict__ pval,
                  float *__restrict__ pval32, double *__restrict__ pdiag,
                  double *__restrict__ prhs, int coarse_mode, const float *__restrict__ hw,
                  const float *__restrict__ emb, const double *__restrict__ logd,
                  double *__restrict__ zd) {
    const int lane = threadIdx.x & 31;
    const int32_t k0 = (static_cast<int32_t>(blockIdx.x) * kPfWarps + (threadIdx.x >> 5)) * 32;
    if (k0 >= rows) return;  // whole warp
    const int32_t k = k0 + lane;
    int32_t c = 0, e0 = 0, len = 0;
    bool yax = false;
    if (k < rows) {
        c = __ldg(order + k);
        const RowRef r = row_of(L, c);
        e0 = r.e0;
        len = r.e1 - r.e0;
        yax = r.off != 0;
    }
    int32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    const int32_t excl = incl - len;
    const int32_t T = __shfl_sync(0xffffffffu, incl, 31);
    const int32_t dst0 = __shfl_sync(0xffffffffu, k < rows ? __ldg(prp + k) : 0, 0);
    for (int32_t t0 = 0; t0 < T; t0 += 32) {
        const int32_t t = t0 + lane;
        int row = 0;  // the last lane whose exclusive offset is <= t
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
            const int cand = row + step;
            const int32_t ex = __shfl_sync(0xffffffffu, excl, cand & 31);
            if (cand < 32 && ex <= t) row = cand;
        }
        const int32_t re0 = __shfl_sync(0xffffffffu, e0, row);
        const int32_t rex = __shfl_sync(0xffffffffu, excl, row);
        const bool ry = __shfl_sync(0xffffffffu, yax, row);
        if (t < T) {
            const int32_t e = re0 + (t - rex);
            const int32_t off = ry ? L.n : 0;
            const int32_t *col = ry ? L.col1 : L.col0;
            const double *val = ry ? L.val1 : L.val0;
            const double v = __ldg(val + e);
            pcol[dst0 + t] = newpos[__ldg(col + e) + off] - off;
            pval[dst0 + t] = v;
            pval32[dst0 + t] = static_cast<float>(v);
        }
    }
    if (k >= rows) return;
    const bool y = yax;
    const int32_t i = y ? c - L.n : c;
    const double d = __ldg((y ? L.diag1 : L.diag0) + i);
    pdiag[k] = d;
    prhs[k] = __ldg((y ? rhs1 : rhs0) + i);
    if (coarse_mode > 0) {  // the coarse vector, rounded to FP32 as the solve uses it
        double z = 1.0;
        if (coarse_mode >= 2) {
            const double *val = y ? L.val1 : L.val0;
            double sabs = 0.0;
            for (int32_t e = e0; e < e0 + len; ++e) sabs += fabs(__ldg(val + e));
            if (coarse_mode == 2)
                z = static_cast<double>(static_cast<float>(sabs / d));
            else  // the learned head on the cell's embedding
                z = static_cast<double>(coarse_head_z(emb + static_cast<int64_t>(i) * kCoarseProj,
                                                      sabs, d, __ldg(logd + (y ? 1 : 0)),
                                                      [&](int t) { return __ldg(hw + t); }));
        }
        zd[k] = z;
    }
}

// Eight lanes per aggregate (lane m holds row m of its block), four
// aggregates per warp, the rows in shared memory (a padded row per lane):
// each lane forms its row of the block of A (the diagonal, then the row's
// entries inside the aggregate in storage order, duplicates summed), the
// group factors B = L L^T in FP64 row by row (the pivot lane takes sqrt and
// one reciprocal; the other lanes read the pivot row from shared memory),
// and lane m then solves L L^T x = e_m by forward and back substitution,
// reading the rows of L it needs: x is column m of B^-1, that is row m,
// written as 8 FP32 (zero past the aggregate's size; two 16-byte stores,
// consecutive lanes on consecutive rows). A non-positive pivot gives the
// aggregate the inverse of its diagonal instead. Rows indexed in shared
// memory rather than as register arrays keep the assembly free of
// compare-and-select chains and the registers low enough for more warps.
constexpr int kInvWarps = 8;
constexpr int kInvPerBlock = kInvWarps * 4;  // aggregates per block
constexpr int kInvStride = kAggMax + 1;      // doubles per row slot (bank spread)
__global__ void __launch_bounds__(32 * kInvWarps)
    k_blockinv_lanes(const int32_t *count, const int32_t *__restrict__ agg_start,
                     const int32_t *__restrict__ size, int32_t n, const int32_t *__restrict__ prp,
                     const int32_t *__restrict__ pcol, const double *__restrict__ pval,
                     const double *__restrict__ pdiag, float *__restrict__ minv,
                     int32_t *__restrict__ meta) {
    __shared__ double rows_s[kInvWarps][32][kInvStride];
    __shared__ double rinv_s[kInvWarps][32];
    __shared__ int ok_s[kInvWarps][4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g0 = lane & ~7;  // first lane of this aggregate's group
    const int m = lane & 7;
    const int32_t J = (static_cast<int32_t>(blockIdx.x) * kInvWarps + w) * 4 + (lane >> 3);
    const int32_t cnt = *count;
    if ((static_cast<int32_t>(blockIdx.x) * kInvWarps + w) * 4 >= cnt) return;  // whole warp
    double (*R)[kInvStride] = rows_s[w] + g0;  // the group's rows
    double *me = rows_s[w][lane];
    double *rv = rinv_s[w] + g0;
    int k = 0;
    int32_t first = 0, first_l = 0;
    if (J < cnt) {
        first = __ldg(agg_start + J);
        k = __ldg(size + J);
        first_l = first >= n ? first - n : first;
    }
    const bool mine = m < k;
#pragma unroll
    for (int t = 0; t < kAggMax; ++t) me[t] = 0.0;
    rv[m] = 0.0;
    if (m == 0) ok_s[w][lane >> 3] = 1;
    double d = 1.0;
    if (mine) {
        const int32_t row = first + m;
        d = __ldg(pdiag + row);
        me[m] += d;
        // four entries per round with independent loads, added in storage order
        const int32_t e1 = __ldg(prp + row + 1);
        for (int32_t e = __ldg(prp + row); e < e1; e += 4) {
            int32_t cq[4];
            double cv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                cq[u] = e + u < e1 ? __ldg(pcol + e + u) - first_l : -1;
                cv[u] = e + u < e1 ? __ldg(pval + e + u) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (cq[u] >= 0 && cq[u] < k) me[cq[u]] += cv[u];
        }
    }
    __syncwarp();
    // Cholesky: row m becomes row m of L (entries past m unused)
    for (int j = 0; j < kAggMax; ++j) {
        if (mine && m == j) {
            double sj = me[j];
            for (int q = 0; q < j; ++q) sj -= me[q] * me[q];
            if (sj > 0.0) {
                me[j] = sqrt(sj);
                rv[j] = 1.0 / me[j];
            } else {
                ok_s[w][lane >> 3] = 0;
            }
        }
        __syncwarp();
        if (mine && m > j) {
            const double *Lj = R[j];
            double u = me[j];
            for (int q = 0; q < j; ++q) u -= me[q] * Lj[q];
            me[j] = u * rv[j];
        }
        __syncwarp();
    }
    const bool ok = ok_s[w][lane >> 3] != 0;
    float out[kAggMax];
    if (ok && mine) {
        // forward: y = L^-1 e_m (y[i] = 0 for i < m)
        double y[kAggMax];
#pragma unroll
        for (int i = 0; i < kAggMax; ++i) {
            const double ri = i < k ? rv[i] : 0.0;
            double acc = 0.0;
#pragma unroll
            for (int q = 0; q < i; ++q) acc += (i < k ? R[i][q] : 0.0) * y[q];
            y[i] = i < m ? 0.0 : (i == m ? ri : -acc * ri);
        }
        // back: x = L^-T y, in place (y[i] is read before x[i] replaces it)
#pragma unroll
        for (int i = kAggMax - 1; i >= 0; --i) {
            const double ri = i < k ? rv[i] : 0.0;
            double acc = y[i];
#pragma unroll
            for (int q = i + 1; q < kAggMax; ++q)
                if (q < k) acc -= R[q][i] * y[q];  // L[q][i]
            y[i] = acc * ri;
        }
#pragma unroll
        for (int t = 0; t < kAggMax; ++t) out[t] = t < k ? static_cast<float>(y[t]) : 0.0f;
    } else {
#pragma unroll
        for (int t = 0; t < kAggMax; ++t) out[t] = t == m ? static_cast<float>(1.0 / d) : 0.0f;
    }
    if (!mine) return;
    float4 *dst = reinterpret_cast<float4 *>(minv + static_cast<size_t>(first + m) * kAggMax);
    dst[0] = make_float4(out[0], out[1], out[2], out[3]);
    dst[1] = make_float4(out[4], out[5], out[6], out[7]);
    meta[first + m] = first_l * kAggMax + (k - 1);
}

// blk_start[b] = first aggregate start >= b * ceil(rows / grid).
__global__ void k_blkstart(int grid, int32_t rows, const int32_t *count, const int32_t *agg_start,
                           int32_t *blk_start) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > grid) return;
    const int32_t per = (rows + grid - 1) / grid;
    const int64_t t64 = static_cast<int64_t>(b) * per;
    const int32_t T = t64 > rows ? rows : static_cast<int32_t>(t64);
    int32_t lo = 0, hi = *count;  // first index with agg_start >= T
    while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (agg_start[mid] < T) lo = mid + 1;
        else hi = mid;
    }
    blk_start[b] = (b == grid || lo >= *count) ? rows : agg_start[lo];
}

__global__ void k_perm_in(int32_t rows, int32_t n, const int32_t *order, const double *x,
                          const double *y, double *px) {
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= rows) return;
    const int32_t c = order[k];
    px[k] = c < n ? x[c] : y[c - n];
}

__global__ void k_perm_out(int32_t rows, int32_t n, const int32_t *order, const double *px,
                           double *x, double *y) {
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= rows) return;
    const int32_t c = order[k];
    if (c < n) x[c] = px[k];
    else y[c - n] = px[k];
}

// ---- coarse correction: z, A z and 1 / (z^T A z) per axis ------------------
//
// The smooth error left by block Jacobi on a SimPL system is dominated by one
// mode: the whole placement moving together (a Laplacian held only by the
// anchors and the fixed pins). The mixed solve removes it with the additive
// coarse term z (z^T A z)^-1 z^T r. z per permuted row:
//   mode 1  the constant 1;
//   mode 2  the share of the row's weight that couples to other movable
//           cells, sum_j |a_ij| / a_ii (cells held only by fixed pins and
//           anchors do not take part in the rigid motion);
//   mode 3  the learned head on the row's cell embedding, its coupling share
//           and its log diagonal (ktg_coarse_head.cuh).
__global__ void k_coarse_z(int mode, int32_t rows, int32_t n, const int32_t *prp,
                           const double *pval, const double *pdiag, const int32_t *order,
                           const float *hw, const float *emb, const double *logd, double *zd) {
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= rows) return;
    float z = 1.0f;
    if (mode >= 2) {
        double sabs = 0.0;
        for (int32_t e = __ldg(prp + k); e < __ldg(prp + k + 1); ++e) sabs += fabs(__ldg(pval + e));
        const double d = __ldg(pdiag + k);
        if (mode == 2) {
            z = static_cast<float>(sabs / d);
        } else {
            const int32_t c = __ldg(order + k);
            const bool y = c >= n;
            z = coarse_head_z(emb + static_cast<int64_t>(y ? c - n : c) * kCoarseProj, sabs, d,
                              __ldg(logd + (y ? 1 : 0)), [&](int t) { return __ldg(hw + t); });
        }
    }
    zd[k] = z;
}

// (A z)_k in FP64 (row sums of a Laplacian-like system cancel: the FP32
// result keeps its relative precision only if it is formed in FP64) as warp
// tiles over the permuted system, stored with z as (z, A z) in FP32; block
// partials of z^T A z per axis, summed in block order by the last block,
// which writes 1 / (z^T A z) (0 when not positive).
constexpr int kAzThreads = 256;
__global__ void __launch_bounds__(kAzThreads)
    k_coarse_az(const int32_t *__restrict__ prp, const int32_t *__restrict__ pcol,
                const double *__restrict__ pval, const double *__restrict__ pdiag,
                const double *__restrict__ zd, int32_t n, int32_t rows_total,
                int32_t rows_per_block, float2 *__restrict__ zaz, double *part, unsigned *ticket,
                double *einv) {
    __shared__ __align__(16) double tilebuf[(kAzThreads / 32) * kTileChunk];
    __shared__ int32_t wb[kAzThreads / 32 + 1];
    __shared__ double red[33 * 2];
    const int32_t r0 = static_cast<int32_t>(blockIdx.x) * rows_per_block;
    const int32_t R = min(rows_per_block, rows_total - r0);
    const int32_t base = __ldg(prp + r0);
    warp_row_bounds(R, wb, [&](int32_t l) {
        return int64_t(__ldg(prp + r0 + l)) - base + int64_t(kRowCost) * l;
    });
    double e[2] = {0.0, 0.0};
    warp_tile_spmv<double>(
        r0, n, R, nullptr, wb, tilebuf,
        [&](int pass, const int32_t *&trp, const int32_t *&tcol, const double *&tval,
            const double *&tin) {
            trp = prp + (pass ? n : 0);
            tcol = pcol;
            tval = pval;
            tin = zd + (pass ? n : 0);
        },
        [&](int32_t l, int, int32_t) { return __ldg(pdiag + r0 + l) * __ldg(zd + r0 + l); },
        [&](int32_t l, int axis, int32_t, double az) {
            const double z = __ldg(zd + r0 + l);
            zaz[r0 + l] = make_float2(static_cast<float>(z), static_cast<float>(az));
            e[axis] += z * az;
        });
    block_sum_k<2>(e, red);
    if (threadIdx.x == 0) {
        __stcg(part + 2 * blockIdx.x, e[0]);
        __stcg(part + 2 * blockIdx.x + 1, e[1]);
    }
    if (last_block_done(ticket)) {
        double t[2] = {0.0, 0.0};
        for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += blockDim.x) {
            t[0] += __ldcg(part + 2 * b);
            t[1] += __ldcg(part + 2 * b + 1);
        }
        block_sum_k<2>(t, red);
        if (threadIdx.x == 0) {
            einv[0] = t[0] > 0.0 ? 1.0 / t[0] : 0.0;
            einv[1] = t[1] > 0.0 ? 1.0 / t[1] : 0.0;
        }
    }
}

template <typename T>
int grow(ktg_ctx *c, T **p, int64_t count) {
    if (*p) cudaFree(*p);
    *p = nullptr;
    if (count <= 0) count = 1;
    if (cudaMalloc(p, sizeof(T) * count) != cudaSuccess)
        return set_error(c, KTG_ERR_NOMEM, "out of device memory (aggregation)");
    return KTG_OK;
}

int reserve(ktg_ctx *c, AggState *s, int64_t rows, int64_t nnz) {
    int rc = KTG_OK;
    if (rows > s->cap_rows) {
        for (int32_t **p : {&s->mate, &s->pick, &s->flag, &s->cid, &s->child0, &s->child1,
                            &s->size_a, &s->size_b, &s->cur, &s->pos, &s->cstart[0], &s->cstart[1],
                            &s->clen[0], &s->clen[1], &s->order, &s->newpos, &s->meta, &s->ea,
                            &s->eb, &s->la})
            if ((rc = grow(c, p, rows))) return rc;
        if ((rc = grow(c, &s->agg_start, rows + 1))) return rc;
        if ((rc = grow(c, &s->prp, rows + 1))) return rc;
        for (double **p : {&s->cdiag[0], &s->cdiag[1], &s->pdiag, &s->prhs, &s->px})
            if ((rc = grow(c, p, rows))) return rc;
        if ((rc = grow(c, &s->minv, rows * kAggMax))) return rc;
        if ((rc = grow(c, &s->zaz, rows))) return rc;
        if ((rc = grow(c, &s->zd, rows))) return rc;
        if ((rc = grow(c, &s->coarse_part, 2 * ((rows + kT - 1) / kT)))) return rc;
        s->tiles_cap = (std::max(rows, nnz) + kScanTile - 1) / kScanTile + 1;
        if ((rc = grow(c, &s->tile_sum, s->tiles_cap))) return rc;
        s->cap_rows = rows;
    }
    if (nnz > s->cap_nnz) {
        for (int t = 0; t < 2; ++t) {
            if ((rc = grow(c, &s->ccol[t], nnz))) return rc;
            if ((rc = grow(c, &s->cval[t], nnz))) return rc;
        }
        if ((rc = grow(c, &s->pcol, nnz))) return rc;
        if ((rc = grow(c, &s->pval, nnz))) return rc;
        if ((rc = grow(c, &s->pval32, nnz))) return rc;
        s->cap_nnz = nnz;
    }
    if (!s->counts && (rc = grow(c, &s->counts, 8))) return rc;
    if (!s->coarse_einv && (rc = grow(c, &s->coarse_einv, 2))) return rc;
    if (!s->ticket) {
        if ((rc = grow(c, &s->ticket, 1))) return rc;
        KTG_CUDA(c, cudaMemsetAsync(s->ticket, 0, sizeof(unsigned), c->stream));
    }
    return KTG_OK;
}

int blocks_for(int64_t items, int threads) {
    return static_cast<int>(std::max<int64_t>(1, (items + threads - 1) / threads));
}

// Exclusive scan of in[0 .. *count) into out, total into *total.
void scan(ktg_ctx *c, AggState *s, const int32_t *in, int32_t *out, const int32_t *count,
          int64_t upper, int32_t *total) {
    const int tiles = blocks_for(upper, kScanTile);
    k_scan_tiles<<<tiles, 1024, 0, c->stream>>>(in, out, count, s->tile_sum);
    k_scan_sums<<<1, 1024, 0, c->stream>>>(s->tile_sum, count, total);
    k_scan_add<<<blocks_for(upper, kT), kT, 0, c->stream>>>(out, count, s->tile_sum);
    c->launches += 3;
}

}  // namespace

void free_agg(ktg_ctx *c) {
    AggState *s = c->agg;
    if (!s) return;
    for (void *p : {(void *)s->mate, (void *)s->pick, (void *)s->flag, (void *)s->cid,
                    (void *)s->child0, (void *)s->child1, (void *)s->size_a, (void *)s->size_b,
                    (void *)s->cur, (void *)s->pos, (void *)s->cstart[0], (void *)s->cstart[1],
                    (void *)s->clen[0], (void *)s->clen[1], (void *)s->ccol[0], (void *)s->ccol[1],
                    (void *)s->cval[0], (void *)s->cval[1], (void *)s->cdiag[0],
                    (void *)s->cdiag[1], (void *)s->counts, (void *)s->tile_sum,
                    (void *)s->agg_start, (void *)s->order, (void *)s->newpos, (void *)s->prp,
                    (void *)s->pcol, (void *)s->pval, (void *)s->pval32, (void *)s->pdiag,
                    (void *)s->prhs, (void *)s->px, (void *)s->minv, (void *)s->meta,
                    (void *)s->blk_start, (void *)s->gslice, (void *)s->ea, (void *)s->eb,
                    (void *)s->la, (void *)s->zaz, (void *)s->zd, (void *)s->coarse_einv,
                    (void *)s->coarse_part, (void *)s->ticket})
        if (p) cudaFree(p);
    delete s;
    c->agg = nullptr;
}

// Builds aggregates, the permuted system and the block inverses for the
// current systems, all on c->stream without host synchronisation (buffers
// grow, with a synchronising cudaMalloc, only when the systems outgrow them).
int build_agg(ktg_ctx *c) {
    if (!c->agg) c->agg = new AggState();
    AggState *s = c->agg;
    const int64_t n = c->sys_n;
    const int64_t rows = 2 * n;
    if (rows > 0x3fffffffll / kAggMax)
        return set_error(c, KTG_ERR_RANGE, "system too large for the aggregation preconditioner");
    const int64_t nnz_cap = 2 * c->sys_cap_nnz;
    int rc = reserve(c, s, rows, nnz_cap);
    if (rc) return rc;
    const int32_t R = static_cast<int32_t>(rows);
    if (rows == 0) {  // counts all zero: empty row ranges for the solve
        k_init<<<1, kT, 0, c->stream>>>(0, s->cur, s->pos, s->size_a, s->mate, s->counts);
        ++c->launches;
        s->blk_grid = 0;
        c->agg_ready = true;
        KTG_CUDA(c, cudaGetLastError());
        return KTG_OK;
    }
    LevelView L0{};
    L0.fine = true;
    L0.n = static_cast<int32_t>(n);
    L0.rp0 = c->sys[0].row_ptr;
    L0.rp1 = c->sys[1].row_ptr;
    L0.col0 = c->sys[0].col;
    L0.col1 = c->sys[1].col;
    L0.val0 = c->sys[0].val;
    L0.val1 = c->sys[1].val;
    L0.diag0 = c->sys[0].diag;
    L0.diag1 = c->sys[1].diag;
    int32_t *cnt = s->counts;  // cnt[l] = nodes at level l; 4, 6, 7 scratch counts
    const int gR = blocks_for(rows, kT);
    k_init<<<gR, kT, 0, c->stream>>>(R, s->cur, s->pos, s->size_a, s->mate, cnt);
    ++c->launches;
    int32_t *size_old = s->size_a, *size_new = s->size_b;
    LevelView L = L0;
    for (int level = 0; level < kLevels; ++level) {
        const int32_t *count = cnt + level;
        // strengths of this level's entries live in cval[level & 1] until this
        // level's coarsening overwrites that buffer (level 0 reads the axis
        // CSRs, level l > 0 reads cval[(l - 1) & 1])
        double *sbuf = s->cval[level & 1];
        const int64_t yoff = c->sys_cap_nnz;
        const int gP = blocks_for(rows, 32 * kPickWarps);
        for (int round = 0; round < kRounds; ++round) {
            if (round == 0)
                k_pick<true><<<gP, 32 * kPickWarps, 0, c->stream>>>(L, count, s->mate, s->pick, sbuf, yoff);
            else
                k_pick<false><<<gP, 32 * kPickWarps, 0, c->stream>>>(L, count, s->mate, s->pick, sbuf, yoff);
            k_handshake<<<gR, kT, 0, c->stream>>>(count, s->pick, s->mate);
            c->launches += 2;
        }
        k_leader_flag<<<gR, kT, 0, c->stream>>>(count, s->mate, s->flag);
        ++c->launches;
        scan(c, s, s->flag, s->flag, count, rows, cnt + level + 1);
        k_number<<<gR, kT, 0, c->stream>>>(count, s->mate, s->flag, s->cid, s->child0, s->child1,
                                           size_old, size_new);
        k_follow<<<gR, kT, 0, c->stream>>>(R, s->cur, s->pos, s->mate, s->cid, size_old);
        c->launches += 2;
        if (level + 1 < kLevels) {
            const int t = level & 1;
            const int32_t *next = cnt + level + 1;
            // raw lengths in s->pick (free until the next level's matching);
            // the heavy-row list in s->flag (its scan was used by k_number)
            k_rawlen<<<gR, kT, 0, c->stream>>>(L, next, s->child0, s->child1, s->pick, s->ea,
                                               s->eb, s->la);
            scan(c, s, s->pick, s->cstart[t], next, rows, cnt + 4);
            KTG_CUDA(c, cudaMemsetAsync(cnt + 7, 0, sizeof(int32_t), c->stream));
            const CoarseArgs CA{L,          next,         s->child0, s->child1,  s->cid,
                                s->cstart[t], s->pick,    s->ea,     s->eb,      s->la,
                                s->clen[t], s->ccol[t],   s->cval[t], s->cdiag[t], s->flag,
                                cnt + 7};
            if (rows < (1ll << 26))
                k_coarse_warp<uint32_t><<<8 * c->num_sms, 32 * kWarpWarps, 0, c->stream>>>(CA);
            else
                k_coarse_warp<unsigned long long><<<8 * c->num_sms, 32 * kWarpWarps, 0, c->stream>>>(CA);
            k_coarse_heavy<<<4 * c->num_sms, kHeavyThreads, 0, c->stream>>>(CA);
            k_reset_mate<<<gR, kT, 0, c->stream>>>(next, s->mate);
            c->launches += 4;
            LevelView C{};
            C.fine = false;
            C.start = s->cstart[t];
            C.len = s->clen[t];
            C.ccol = s->ccol[t];
            C.cval = s->cval[t];
            C.cdiag = s->cdiag[t];
            L = C;
        }
        std::swap(size_old, size_new);
    }
    // size_old now holds the aggregate sizes; cnt[kLevels] the aggregate count
    const int32_t *nagg = cnt + kLevels;
    scan(c, s, size_old, s->agg_start, nagg, rows, cnt + 5);
    k_newpos<<<gR, kT, 0, c->stream>>>(R, s->cur, s->pos, s->agg_start, s->newpos, s->order);
    ++c->launches;
    KTG_CUDA(c, cudaGetLastError());
    s->final_size = size_old;
    s->struct_rows = rows;
    s->struct_gen = c->netlist_gen;
    s->blk_grid = 0;  // row ranges follow the new aggregates
    s->builds_on_struct = 0;
    return build_agg_values(c);
}

// The numeric part for the current systems on the aggregates in place
// (the row order, the aggregates' sizes and starts): the permuted system and
// its FP32 copy, the block inverses and the coarse vector's z.
int build_agg_values(ktg_ctx *c) {
    AggState *s = c->agg;
    const int64_t n = c->sys_n;
    const int64_t rows = 2 * n;
    const int32_t R = static_cast<int32_t>(rows);
    if (rows == 0) {
        c->agg_ready = true;
        return KTG_OK;
    }
    const int gR = blocks_for(rows, kT);
    LevelView L0{};
    L0.fine = true;
    L0.n = static_cast<int32_t>(n);
    L0.rp0 = c->sys[0].row_ptr;
    L0.rp1 = c->sys[1].row_ptr;
    L0.col0 = c->sys[0].col;
    L0.col1 = c->sys[1].col;
    L0.val0 = c->sys[0].val;
    L0.val1 = c->sys[1].val;
    L0.diag0 = c->sys[0].diag;
    L0.diag1 = c->sys[1].diag;
    int32_t *cnt = s->counts;
    const int32_t *nagg = cnt + kLevels;
    k_plen<<<gR, kT, 0, c->stream>>>(L0, R, s->order, s->prp);
    ++c->launches;
    // prp: exclusive scan of the permuted row lengths (cnt[6] = R), total at prp[R]
    scan(c, s, s->prp, s->prp, cnt + 6, rows, s->prp + R);
    // the coarse vector of the current mode comes with the permuted system
    // (the learned one only when it is ready)
    const int zmode = (c->coarse == 3 && !c->coarse_z_ready) ? 0 : c->coarse;
    k_pfill_tiles<<<blocks_for(rows, 32 * kPfWarps), 32 * kPfWarps, 0, c->stream>>>(
        L0, R, s->order, s->newpos, s->prp, c->sys[0].rhs, c->sys[1].rhs, s->pcol, s->pval,
        s->pval32, s->pdiag, s->prhs, zmode, c->coarse_head_w, c->coarse_emb, c->coarse_logd,
        s->zd);
    k_blockinv_lanes<<<blocks_for(rows, kInvPerBlock), 32 * kInvWarps, 0, c->stream>>>(
        nagg, s->agg_start, s->final_size, static_cast<int32_t>(n), s->prp, s->pcol, s->pval,
        s->pdiag, s->minv, s->meta);
    c->launches += 2;
    KTG_CUDA(c, cudaGetLastError());
    s->coarse_mode = 0;
    s->z_mode = zmode;  // z of this mode is in s->zd; A z not formed yet
    s->z_gen = c->coarse_z_gen;
    c->agg_ready = true;
    return KTG_OK;
}

// The aggregation preconditioner for the current systems: the whole build,
// or, with the "agg_reuse" option K > 0, the numeric part alone on the
// aggregates of an earlier build of the same netlist for up to K builds in a
// row (SimPL's systems change little from one global iteration to the next;
// the cell grouping stays good while the values are taken afresh).
int prepare_agg(ktg_ctx *c) {
    AggState *s = c->agg;
    const bool reuse = c->agg_reuse > 0 && s && s->struct_rows == 2 * c->sys_n &&
                       s->struct_gen == c->netlist_gen && s->builds_on_struct < c->agg_reuse &&
                       s->cap_nnz >= 2 * c->sys_cap_nnz;
    if (!reuse) return build_agg(c);
    ++s->builds_on_struct;
    return build_agg_values(c);
}

// The coarse vector of `mode` (1, 2, or 3 with zin) for the current
// aggregates and its A z and 1 / (z^T A z); kept until the next build.
int agg_coarse_setup(ktg_ctx *c, int mode) {
    AggState *s = c->agg;
    const int64_t rows = 2 * c->sys_n;
    if (!s || !c->agg_ready) return set_error(c, KTG_ERR_STATE, "no aggregates to correct");
    if (mode == 3 && (!c->coarse_z_ready || !c->coarse_head_w))
        return set_error(c, KTG_ERR_STATE, "no learned coarse vector");
    if (s->coarse_mode == mode && (mode != 3 || s->z_gen == c->coarse_z_gen)) return KTG_OK;
    if (rows == 0) {
        KTG_CUDA(c, cudaMemsetAsync(s->coarse_einv, 0, 2 * sizeof(double), c->stream));
        s->coarse_mode = mode;
        return KTG_OK;
    }
    const int32_t R = static_cast<int32_t>(rows), n = static_cast<int32_t>(c->sys_n);
    if (s->z_mode != mode || (mode == 3 && s->z_gen != c->coarse_z_gen)) {  // z is stale
        k_coarse_z<<<blocks_for(rows, kT), kT, 0, c->stream>>>(
            mode, R, n, s->prp, s->pval, s->pdiag, s->order, c->coarse_head_w, c->coarse_emb,
            c->coarse_logd, s->zd);
        ++c->launches;
        s->z_mode = mode;
        s->z_gen = c->coarse_z_gen;
    }
    // one even wave of 256-thread blocks (6 per SM), at least 256 rows each
    const int64_t slots = 6ll * c->num_sms;
    const int32_t per = static_cast<int32_t>(std::max<int64_t>(256, (rows + slots - 1) / slots));
    const int blocks = static_cast<int>((rows + per - 1) / per);
    if (2 * blocks > 2 * ((rows + kT - 1) / kT))
        return set_error(c, KTG_ERR_STATE, "coarse partials buffer too small");
    k_coarse_az<<<blocks, kAzThreads, 0, c->stream>>>(s->prp, s->pcol, s->pval, s->pdiag, s->zd, n,
                                                      R, per, s->zaz, s->coarse_part, s->ticket,
                                                      s->coarse_einv);
    ++c->launches;
    KTG_CUDA(c, cudaGetLastError());
    s->coarse_mode = mode;
    return KTG_OK;
}

// Row ranges of the persistent kernel's blocks aligned to aggregates, and a
// permuted copy of the positions; returns the per-block slice capacity.
int agg_prepare_solve(ktg_ctx *c, int grid, const double *x, const double *y, int32_t *rows_cap) {
    AggState *s = c->agg;
    const int64_t rows = 2 * c->sys_n;
    if (s->blk_grid != grid) {
        if (grid + 1 > s->grid_cap) {
            int rc = grow(c, &s->blk_start, grid + 1);
            if (rc) return rc;
            s->grid_cap = grid + 1;
        }
        k_blkstart<<<blocks_for(grid + 1, kT), kT, 0, c->stream>>>(
            grid, static_cast<int32_t>(rows), s->counts + kLevels, s->agg_start, s->blk_start);
        ++c->launches;
        s->blk_grid = grid;
    }
    *rows_cap = static_cast<int32_t>((rows + grid - 1) / grid + kAggMax);
    if (rows > 0) {
        k_perm_in<<<blocks_for(rows, kT), kT, 0, c->stream>>>(
            static_cast<int32_t>(rows), static_cast<int32_t>(c->sys_n), s->order, x, y, s->px);
        ++c->launches;
    }
    KTG_CUDA(c, cudaGetLastError());
    return KTG_OK;
}

int agg_finish_solve(ktg_ctx *c, double *x, double *y) {
    AggState *s = c->agg;
    const int64_t rows = 2 * c->sys_n;
    if (rows > 0) {
        k_perm_out<<<blocks_for(rows, kT), kT, 0, c->stream>>>(
            static_cast<int32_t>(rows), static_cast<int32_t>(c->sys_n), s->order, s->px, x, y);
        ++c->launches;
    }
    KTG_CUDA(c, cudaGetLastError());
    return KTG_OK;
}

double *agg_global_slices(ktg_ctx *c, int64_t doubles) {
    AggState *s = c->agg ? c->agg : (c->agg = new AggState());
    if (doubles > s->gslice_cap) {
        if (grow(c, &s->gslice, doubles)) return nullptr;
        s->gslice_cap = doubles;
    }
    return s->gslice;
}

}  // namespace ktg
