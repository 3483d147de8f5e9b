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
#include "ktg_common.cuh"
#include "ktg_context.h"

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

// One thread per node, four entries of its row fetched at a time so that
// their gathers (mate and diag of the neighbour) are in flight together. Rows
// longer than kPickShort are queued in shared memory and scanned afterwards
// by a whole warp each, so the long tail of row lengths does not set the
// kernel's time. The result (largest strength, ties to the smaller J) does
// not depend on the order of the scan.
constexpr int kPickShort = 16;
constexpr int kPickThreads = 256;

__device__ __forceinline__ void pick_consider(int32_t I, int32_t J, double v, double dI,
                                              double dJ, int32_t mJ, double &best, int32_t &bj) {
    if (J == I || mJ >= 0) return;
    const double s = -v / sqrt(dI * dJ);
    if (s > 0.0 && (s > best || (s == best && J < bj))) {
        best = s;
        bj = J;
    }
}

__device__ __forceinline__ void pick_merge(double ob, int32_t oj, double &best, int32_t &bj) {
    if (oj >= 0 && (bj < 0 || ob > best || (ob == best && oj < bj))) {
        best = ob;
        bj = oj;
    }
}

__global__ void __launch_bounds__(kPickThreads) k_pick(LevelView L, const int32_t *count,
                                                       const int32_t *mate, int32_t *pick) {
    __shared__ int32_t queue[kPickThreads];
    __shared__ int qn;
    if (threadIdx.x == 0) qn = 0;
    __syncthreads();
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    const int32_t cnt = *count;
    if (I < cnt) {
        if (mate[I] >= 0) {
            pick[I] = -1;
        } else {
            const RowRef r = row_of(L, I);
            if (r.e1 - r.e0 > kPickShort) {
                queue[atomicAdd(&qn, 1)] = I;
            } else {
                const double dI = diag_of(L, I);
                double best = 0.0;
                int32_t bj = -1;
                int32_t e = r.e0;
                for (; e + 4 <= r.e1; e += 4) {
                    int32_t J[4], mJ[4];
                    double v[4], dJ[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        J[q] = __ldg(r.col + e + q) + r.off;
                        v[q] = __ldg(r.val + e + q);
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        mJ[q] = mate[J[q]];
                        dJ[q] = diag_of(L, J[q]);
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) pick_consider(I, J[q], v[q], dI, dJ[q], mJ[q], best, bj);
                }
                for (; e < r.e1; ++e) {
                    const int32_t J = __ldg(r.col + e) + r.off;
                    pick_consider(I, J, __ldg(r.val + e), dI, diag_of(L, J), mate[J], best, bj);
                }
                pick[I] = bj;
            }
        }
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = w; q < qn; q += kPickThreads / 32) {
        const int32_t node = queue[q];
        const RowRef r = row_of(L, node);
        const double dI = diag_of(L, node);
        double best = 0.0;
        int32_t bj = -1;
        for (int32_t e = r.e0 + lane; e < r.e1; e += 32) {
            const int32_t J = __ldg(r.col + e) + r.off;
            pick_consider(node, J, __ldg(r.val + e), dI, diag_of(L, J), mate[J], best, bj);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int32_t oj = __shfl_xor_sync(0xffffffffu, bj, o);
            pick_merge(ob, oj, best, bj);
        }
        if (lane == 0) pick[node] = bj;
    }
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

__global__ void k_rawlen(LevelView L, const int32_t *count, const int32_t *child0,
                         const int32_t *child1, int32_t *rawlen) {
    const int32_t J = blockIdx.x * blockDim.x + threadIdx.x;
    if (J >= *count) return;
    const RowRef ra = row_of(L, child0[J]);
    int32_t len = ra.e1 - ra.e0;
    const int32_t b = child1[J];
    if (b >= 0) {
        const RowRef rb = row_of(L, b);
        len += rb.e1 - rb.e0;
    }
    rawlen[J] = len;
}

// Coarse row J = (a, b): the raw entries (row a's, then row b's) mapped to
// coarse ids; ids equal to J fold into the diagonal in raw order
// (d_a, a's entries, d_b, b's entries); the others are summed per id in raw
// order and stored with the ids ascending. Two persistent grid-stride kernels:
//   k_coarse_light: one thread per row of raw length R <= kLight, sorted
//     insertion into a per-thread list in shared memory, entries fetched
//     eight at a time; longer rows are appended to a list (order free: each
//     row is processed on its own);
//   k_coarse_heavy: one warp per listed row: bitonic sort of (id, raw index)
//     in shared memory for R <= kHeavyMax, else sorted insertion by one lane
//     directly in the output row (rare: rows that long need nets of hundreds
//     of pins).
constexpr int kLight = 32;
constexpr int kLightThreads = 128;
constexpr int kHeavyMax = 1024;
constexpr int kHeavyWarps = 4;
constexpr size_t kHeavySmem = static_cast<size_t>(kHeavyWarps) * kHeavyMax * 16;

struct CoarseArgs {
    LevelView L;
    const int32_t *count;
    const int32_t *child0, *child1, *cid, *start, *rawlen;
    int32_t *out_len, *out_col;
    double *out_val, *out_diag;
    int32_t *heavy;        // rows with R > kLight
    int32_t *heavy_count;  // zero before k_coarse_light
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

__global__ void __launch_bounds__(kLightThreads) k_coarse_light(CoarseArgs A) {
    __shared__ int32_t keys_s[kLight * kLightThreads];
    __shared__ double sums_s[kLight * kLightThreads];
    constexpr int T = kLightThreads;
    int32_t *keys = keys_s + threadIdx.x;  // entry q at keys[q * T]
    double *sums = sums_s + threadIdx.x;
    const LevelView &L = A.L;
    const int32_t cnt = *A.count;
    for (int32_t J = blockIdx.x * blockDim.x + threadIdx.x; J < cnt; J += gridDim.x * blockDim.x) {
        const int32_t R = A.rawlen[J];
        if (R > kLight) {
            A.heavy[atomicAdd(A.heavy_count, 1)] = J;
            continue;
        }
        const int32_t a = A.child0[J], b = A.child1[J];
        const RowRef ra = row_of(L, a);
        const int la = ra.e1 - ra.e0;
        RowRef rb = ra;
        if (b >= 0) rb = row_of(L, b);
        double dacc = diag_of(L, a);
        int k = 0;
        for (int e0 = 0; e0 < R; e0 += 8) {
            int32_t K[8];
            double v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int e = e0 + q;
                K[q] = -1;
                v[q] = 0.0;
                if (e < R) {
                    const bool in_a = e < la;
                    const int32_t idx = in_a ? ra.e0 + e : rb.e0 + (e - la);
                    const int32_t c = __ldg((in_a ? ra.col : rb.col) + idx) + (in_a ? ra.off : rb.off);
                    v[q] = __ldg((in_a ? ra.val : rb.val) + idx);
                    K[q] = c;
                }
            }
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (e0 + q < R) K[q] = A.cid[K[q]];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int e = e0 + q;
                if (e >= R) break;
                if (e == la) dacc += diag_of(L, b);
                if (K[q] == J) dacc += v[q];
                else sorted_add(keys, sums, T, k, K[q], v[q]);
            }
        }
        if (la == R && b >= 0) dacc += diag_of(L, b);
        int32_t *oc = A.out_col + A.start[J];
        double *ov = A.out_val + A.start[J];
        for (int q = 0; q < k; ++q) {
            oc[q] = keys[q * T];
            ov[q] = sums[q * T];
        }
        A.out_len[J] = k;
        A.out_diag[J] = dacc;
    }
}

__global__ void __launch_bounds__(32 * kHeavyWarps) k_coarse_heavy(CoarseArgs A) {
    extern __shared__ unsigned long long heavy_smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long *key = heavy_smem + static_cast<size_t>(w) * kHeavyMax * 2;
    double *vr = reinterpret_cast<double *>(key + kHeavyMax);
    const LevelView &L = A.L;
    const int32_t nh = *A.heavy_count;
    for (int32_t h = blockIdx.x * kHeavyWarps + w; h < nh; h += gridDim.x * kHeavyWarps) {
        const int32_t J = A.heavy[h];
        const int32_t R = A.rawlen[J];
        const int32_t a = A.child0[J], b = A.child1[J];
        const RowRef ra = row_of(L, a);
        const int la = ra.e1 - ra.e0;
        RowRef rb = ra;
        if (b >= 0) rb = row_of(L, b);
        if (R > kHeavyMax) {
            if (lane == 0) {
                int32_t *keys = A.out_col + A.start[J];
                double *sums = A.out_val + A.start[J];
                int k = 0;
                double dacc = diag_of(L, a);
                for (int e = 0; e < R; ++e) {
                    if (e == la) dacc += diag_of(L, b);
                    const bool in_a = e < la;
                    const int32_t idx = in_a ? ra.e0 + e : rb.e0 + (e - la);
                    const int32_t K =
                        A.cid[__ldg((in_a ? ra.col : rb.col) + idx) + (in_a ? ra.off : rb.off)];
                    const double v = __ldg((in_a ? ra.val : rb.val) + idx);
                    if (K == J) dacc += v;
                    else sorted_add(keys, sums, 1, k, K, v);
                }
                if (la == R && b >= 0) dacc += diag_of(L, b);
                A.out_len[J] = k;
                A.out_diag[J] = dacc;
            }
            __syncwarp();
            continue;
        }
        int P = 1;
        while (P < R) P <<= 1;
        for (int e = lane; e < P; e += 32) {
            if (e < R) {
                const bool in_a = e < la;
                const int32_t idx = in_a ? ra.e0 + e : rb.e0 + (e - la);
                const int32_t K =
                    A.cid[__ldg((in_a ? ra.col : rb.col) + idx) + (in_a ? ra.off : rb.off)];
                key[e] = (static_cast<unsigned long long>(static_cast<uint32_t>(K)) << 32) |
                         static_cast<uint32_t>(e);
                vr[e] = __ldg((in_a ? ra.val : rb.val) + idx);
            } else {
                key[e] = ~0ull;
            }
        }
        __syncwarp();
        for (int kk = 2; kk <= P; kk <<= 1) {
            for (int j = kk >> 1; j > 0; j >>= 1) {
                for (int i = lane; i < P; i += 32) {
                    const int ixj = i ^ j;
                    if (ixj > i) {
                        const unsigned long long x = key[i], y = key[ixj];
                        if ((x > y) == ((i & kk) == 0)) {
                            key[i] = y;
                            key[ixj] = x;
                        }
                    }
                }
                __syncwarp();
            }
        }
        // segment heads (ids != J) in ascending order, numbered by a warp scan
        const uint32_t uJ = static_cast<uint32_t>(J);
        int base = 0;
        bool any_diag = false;
        for (int i0 = 0; i0 < R; i0 += 32) {
            const int i = i0 + lane;
            bool head = false, dhead = false;
            uint32_t K = 0;
            if (i < R) {
                K = static_cast<uint32_t>(key[i] >> 32);
                const bool first = i == 0 || static_cast<uint32_t>(key[i - 1] >> 32) != K;
                head = first && K != uJ;
                dhead = first && K == uJ;
            }
            const unsigned hm = __ballot_sync(0xffffffffu, head);
            any_diag = any_diag || __any_sync(0xffffffffu, dhead);
            if (head) {
                const int pos = base + __popc(hm & ((1u << lane) - 1u));
                double sum = vr[static_cast<uint32_t>(key[i])];
                for (int j = i + 1; j < R && static_cast<uint32_t>(key[j] >> 32) == K; ++j)
                    sum += vr[static_cast<uint32_t>(key[j])];
                A.out_col[A.start[J] + pos] = static_cast<int32_t>(K);
                A.out_val[A.start[J] + pos] = sum;
            }
            if (dhead) {
                double dacc = diag_of(L, a);
                bool added_b = false;
                for (int j = i; j < R && static_cast<uint32_t>(key[j] >> 32) == K; ++j) {
                    const uint32_t idx = static_cast<uint32_t>(key[j]);
                    if (!added_b && static_cast<int>(idx) >= la) {
                        dacc += diag_of(L, b);
                        added_b = true;
                    }
                    dacc += vr[idx];
                }
                if (!added_b && b >= 0) dacc += diag_of(L, b);
                A.out_diag[J] = dacc;
            }
            base += __popc(hm);
        }
        if (lane == 0) {
            A.out_len[J] = base;
            if (!any_diag) A.out_diag[J] = b >= 0 ? diag_of(L, a) + diag_of(L, b) : diag_of(L, a);
        }
        __syncwarp();
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

// One thread per permuted row (several rows' gathers in flight per warp):
// columns renumbered (per-axis local), values in FP64 and FP32, diag and rhs
// moved.
__global__ void k_pfill(LevelView L, int32_t rows, const int32_t *order, const int32_t *newpos,
                        const int32_t *prp, const double *rhs0, const double *rhs1,
                        int32_t *pcol, double *pval, float *pval32, double *pdiag,
                        double *prhs) {
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= rows) return;
    const int32_t c = order[k];
    const bool y = c >= L.n;
    const int32_t i = y ? c - L.n : c;
    const RowRef r = row_of(L, c);
    const int32_t off = y ? L.n : 0;
    int32_t *dc = pcol + prp[k] - r.e0;
    double *dv = pval + prp[k] - r.e0;
    float *dv32 = pval32 + prp[k] - r.e0;
    int32_t e = r.e0;
    for (; e + 4 <= r.e1; e += 4) {
        int32_t col[4];
        double v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            col[q] = __ldg(r.col + e + q);
            v[q] = __ldg(r.val + e + q);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) col[q] = newpos[col[q] + off] - off;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            dc[e + q] = col[q];
            dv[e + q] = v[q];
            dv32[e + q] = static_cast<float>(v[q]);
        }
    }
    for (; e < r.e1; ++e) {
        const double v = __ldg(r.val + e);
        dc[e] = newpos[__ldg(r.col + e) + off] - off;
        dv[e] = v;
        dv32[e] = static_cast<float>(v);
    }
    pdiag[k] = __ldg((y ? L.diag1 : L.diag0) + i);
    prhs[k] = __ldg((y ? rhs1 : rhs0) + i);
}

// Eight lanes per aggregate, lane m owning row m of the block: the block
// row from the permuted CSR, a row-oriented Cholesky B = L L^T in FP64 with
// the finished rows broadcast by shuffles, L^-1 by forward substitution and
// inv = L^-T L^-1, written as 8 floats per row. All arrays are indexed by
// compile-time constants, so they stay in registers.
__global__ void __launch_bounds__(256) k_blockinv(const int32_t *count, const int32_t *agg_start,
                                                  const int32_t *size, int32_t n,
                                                  const int32_t *prp, const int32_t *pcol,
                                                  const double *pval, const double *pdiag,
                                                  float *minv, int32_t *meta) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int32_t J = static_cast<int32_t>(t / kAggMax);
    const int m = threadIdx.x & (kAggMax - 1);
    const bool validJ = J < *count;
    int32_t first = 0;
    int k = 1;
    if (validJ) {
        first = agg_start[J];
        k = size[J];
    }
    const bool act = validJ && m < k;
    const int32_t first_l = first >= n ? first - n : first;
    double l[kAggMax];
#pragma unroll
    for (int q = 0; q < kAggMax; ++q) l[q] = 0.0;
    if (act) {
        const int32_t row = first + m;
        const double d = pdiag[row];
#pragma unroll
        for (int q = 0; q < kAggMax; ++q)
            if (q == m) l[q] += d;
        const int32_t e0 = prp[row], e1 = prp[row + 1];
        int32_t e = e0;
        for (; e + 4 <= e1; e += 4) {
            int32_t qe[4];
            double v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                qe[u] = pcol[e + u] - first_l;
                v[u] = pval[e + u];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int32_t qq = qe[u] < k ? qe[u] : -1;
#pragma unroll
                for (int q = 0; q < kAggMax; ++q) l[q] += q == qq ? v[u] : 0.0;
            }
        }
        for (; e < e1; ++e) {
            const int32_t qe = pcol[e] - first_l;
            const int32_t qq = qe < k ? qe : -1;
            const double v = pval[e];
#pragma unroll
            for (int q = 0; q < kAggMax; ++q) l[q] += q == qq ? v : 0.0;
        }
    }
    // Cholesky: after step j, lane j holds L[j][0..j] and lanes i > j hold L[i][j].
    bool ok = true;
#pragma unroll
    for (int j = 0; j < kAggMax; ++j) {
        if (m == j && act) {
            double s = l[j];
#pragma unroll
            for (int q = 0; q < j; ++q) s -= l[q] * l[q];
            ok = s > 0.0;
            l[j] = ok ? sqrt(s) : 1.0;
        }
        double rj[kAggMax];
#pragma unroll
        for (int q = 0; q <= j; ++q) rj[q] = __shfl_sync(0xffffffffu, l[q], j, kAggMax);
        if (act && m > j && j < k) {
            double u = l[j];
#pragma unroll
            for (int q = 0; q < j; ++q) u -= l[q] * rj[q];
            l[j] = u / rj[j];
        }
    }
    const unsigned bad = __ballot_sync(0xffffffffu, !ok);
    const bool group_ok = ((bad >> (threadIdx.x & 31 & ~(kAggMax - 1))) & 0xffu) == 0u;
    // L^-1, row m in li; acc[c] = sum over finished rows t < m of L[m][t] Li[t][c]
    double li[kAggMax], acc[kAggMax];
#pragma unroll
    for (int q = 0; q < kAggMax; ++q) {
        li[q] = 0.0;
        acc[q] = 0.0;
    }
#pragma unroll
    for (int r = 0; r < kAggMax; ++r) {
        if (m == r && act) {
#pragma unroll
            for (int c = 0; c <= r; ++c) li[c] = ((c == r ? 1.0 : 0.0) - acc[c]) / l[r];
        }
        double rt[kAggMax];
#pragma unroll
        for (int c = 0; c <= r; ++c) rt[c] = __shfl_sync(0xffffffffu, li[c], r, kAggMax);
        if (act && m > r && r < k) {
#pragma unroll
            for (int c = 0; c <= r; ++c) acc[c] += l[r] * rt[c];
        }
    }
    // inv row m = sum over t of Li[t][m] * Li[t][.]
    double inv[kAggMax];
#pragma unroll
    for (int q = 0; q < kAggMax; ++q) inv[q] = 0.0;
#pragma unroll
    for (int r = 0; r < kAggMax; ++r) {
        double rt[kAggMax];
#pragma unroll
        for (int c = 0; c <= r; ++c) rt[c] = __shfl_sync(0xffffffffu, li[c], r, kAggMax);
        if (act && r < k) {
            double tm = 0.0;
#pragma unroll
            for (int c = 0; c <= r; ++c)
                if (c == m) tm = rt[c];
#pragma unroll
            for (int c = 0; c <= r; ++c) inv[c] += tm * rt[c];
        }
    }
    if (!act) return;
    float *dst = minv + static_cast<size_t>(first + m) * kAggMax;
    const double dm = 1.0 / pdiag[first + m];
#pragma unroll
    for (int q = 0; q < kAggMax; ++q) {
        const double v = group_ok ? inv[q] : (q == m ? dm : 0.0);
        dst[q] = q < k ? static_cast<float>(v) : 0.0f;
    }
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
                            &s->clen[0], &s->clen[1], &s->order, &s->newpos, &s->meta})
            if ((rc = grow(c, p, rows))) return rc;
        if ((rc = grow(c, &s->agg_start, rows + 1))) return rc;
        if ((rc = grow(c, &s->prp, rows + 1))) return rc;
        for (double **p : {&s->cdiag[0], &s->cdiag[1], &s->pdiag, &s->prhs, &s->px})
            if ((rc = grow(c, p, rows))) return rc;
        if ((rc = grow(c, &s->minv, rows * kAggMax))) return rc;
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
                    (void *)s->blk_start, (void *)s->gslice})
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
    static bool attr_set = false;
    if (!attr_set) {
        KTG_CUDA(c, cudaFuncSetAttribute(k_coarse_heavy, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kHeavySmem)));
        attr_set = true;
    }
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
        for (int round = 0; round < kRounds; ++round) {
            k_pick<<<blocks_for(rows, kPickThreads), kPickThreads, 0, c->stream>>>(L, count, s->mate,
                                                                                   s->pick);
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
            k_rawlen<<<gR, kT, 0, c->stream>>>(L, next, s->child0, s->child1, s->pick);
            scan(c, s, s->pick, s->cstart[t], next, rows, cnt + 4);
            KTG_CUDA(c, cudaMemsetAsync(cnt + 7, 0, sizeof(int32_t), c->stream));
            const CoarseArgs CA{L,          next,        s->child0,   s->child1,
                                s->cid,     s->cstart[t], s->pick,    s->clen[t],
                                s->ccol[t], s->cval[t],  s->cdiag[t], s->flag,
                                cnt + 7};
            k_coarse_light<<<4 * c->num_sms, kLightThreads, 0, c->stream>>>(CA);
            k_coarse_heavy<<<3 * c->num_sms, 32 * kHeavyWarps, kHeavySmem, c->stream>>>(CA);
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
    k_plen<<<gR, kT, 0, c->stream>>>(L0, R, s->order, s->prp);
    c->launches += 2;
    // prp: exclusive scan of the permuted row lengths (cnt[6] = R), total at prp[R]
    scan(c, s, s->prp, s->prp, cnt + 6, rows, s->prp + R);
    k_pfill<<<gR, kT, 0, c->stream>>>(L0, R, s->order, s->newpos, s->prp, c->sys[0].rhs,
                                      c->sys[1].rhs, s->pcol, s->pval, s->pval32, s->pdiag,
                                      s->prhs);
    k_blockinv<<<blocks_for(rows * kAggMax, 256), 256, 0, c->stream>>>(
        nagg, s->agg_start, size_old, static_cast<int32_t>(n), s->prp, s->pcol, s->pval, s->pdiag,
        s->minv, s->meta);
    c->launches += 2;
    KTG_CUDA(c, cudaGetLastError());
    s->blk_grid = 0;  // row ranges follow the new aggregates
    c->agg_ready = true;
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
