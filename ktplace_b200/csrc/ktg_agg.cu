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
// sums in fixed orders, numbering by prefix sums.
//
// Level rules (one level = matching of the level's nodes; the nodes of level
// 0 are the rows, a node of level l + 1 is a matched pair or a single node of
// level l, so it holds at most 2^(l+1) rows):
//   dc(N): the node's Galerkin diagonal, the sum over its member rows m in
//     position order of t_m = d_m + (m's entries whose column lies in N, in
//     storage order); dc = d at level 0;
//   strength of a stored entry (i, j, v) between nodes A (of i) != B (of j):
//     s = -v / sqrt(dc(A) dc(B));
//   kRounds handshake rounds: each unmatched A picks the unmatched B of
//     largest s > 0 over all its member rows' entries (ties: smaller B);
//     mutual picks are matched;
//   leaders (unmatched, or the smaller of a pair) are numbered in order; a
//     row of the second node of a pair moves behind the first's rows.
// The nodes' couplings are the strongest single entries between them, so no
// coarse matrix is formed: a level reads the fine entries with the node of
// each column.
//
// Device memory (per context, grown with the systems): per-node and per-row
// level arrays over 2n, the strength and neighbour node of every fine entry,
// and the permuted system (row_ptr, col, FP64 and FP32 values, diag, rhs, x)
// plus the block inverses (8 floats per row).

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

// The two axis CSRs of the combined row space. Axis arrays are separate
// fields chosen with a conditional, so that no thread copies the parameter
// block to local memory.
struct LevelView {
    int32_t n;  // rows per axis
    const int32_t *rp0, *rp1;
    const int32_t *col0, *col1;
    const double *val0, *val1;
    const double *diag0, *diag1;
};

struct RowRef {
    int32_t e0, e1, off;
    const int32_t *col;
    const double *val;
};

__device__ __forceinline__ RowRef row_of(const LevelView &L, int32_t I) {
    RowRef r;
    const bool y = I >= L.n;
    const int32_t i = y ? I - L.n : I;
    const int32_t *rp = y ? L.rp1 : L.rp0;
    r.e0 = __ldg(rp + i);
    r.e1 = __ldg(rp + i + 1);
    r.off = y ? L.n : 0;
    r.col = y ? L.col1 : L.col0;
    r.val = y ? L.val1 : L.val0;
    return r;
}

__device__ __forceinline__ double diag_of(const LevelView &L, int32_t I) {
    const bool y = I >= L.n;
    return __ldg((y ? L.diag1 : L.diag0) + (y ? I - L.n : I));
}

__global__ void k_init(int32_t rows, int32_t *cur, int32_t *pos, int32_t *size, int32_t *mate,
                       int32_t *counts) {
    pdl_enter();
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

// Level 0, where the nodes are the rows. kFirst (first round of a level:
// nothing is matched yet): computes every entry's strength and stores it in
// sbuf (y rows at offset yoff); later rounds read it back and gather only the
// neighbour's mate.
template <bool kFirst>
__global__ void __launch_bounds__(32 * kPickWarps) k_pick(LevelView L, const int32_t *count,
                                                          const int32_t *mate, int32_t *pick,
                                                          double *sbuf, int64_t yoff) {
    pdl_enter();
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
            const int32_t *col = ry ? L.col1 : L.col0;
            const int32_t J = __ldg(col + e) + (ry ? L.n : 0);
            double *sp = sbuf + (ry ? yoff : 0) + e;
            double st;
            if (kFirst) {
                const double *val = ry ? L.val1 : L.val0;
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

// Levels 1 and up: the same walk over the fine rows whose node is
// unmatched, each entry's column mapped to its node B (cur) and B's diagonal
// (dcr, the diagonal of each row's node: two independent gathers); every
// row's best entry to another unmatched node goes to (cand_s, cand_b), and
// k_nodepick takes the best over a node's member rows. kFirst stores each
// entry's strength and B (sbuf, bbuf) for the level's later rounds.
template <bool kFirst>
__global__ void __launch_bounds__(32 * kPickWarps) k_rowpick(LevelView L, int32_t rows,
                                                             const int32_t *cur,
                                                             const int32_t *mate, const double *dcr,
                                                             double *sbuf, int32_t *bbuf,
                                                             int64_t yoff, double *cand_s,
                                                             int32_t *cand_b) {
    pdl_enter();
    __shared__ double best_s[kPickWarps][32];
    __shared__ int32_t best_j[kPickWarps][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int32_t base = (blockIdx.x * kPickWarps + w) * 32;
    if (base >= rows) return;  // whole warp
    const int32_t I = base + lane;
    bool act = false, yax = false;
    int32_t e0 = 0, len = 0, A = -1;
    double dA = 1.0;
    if (I < rows) {
        A = cur[I];
        if (kFirst || mate[A] < 0) {
            act = true;
            const RowRef r = row_of(L, I);
            e0 = r.e0;
            len = r.e1 - r.e0;
            yax = r.off != 0;
            if (kFirst) dA = dcr[I];
        }
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
        const double rd = __shfl_sync(0xffffffffu, dA, row);
        const int32_t rA = __shfl_sync(0xffffffffu, A, row);
        double sv = 0.0;
        int32_t sj = -1;
        if (t < T) {
            const int32_t e = re0 + (t - rex);
            const int64_t ei = (ry ? yoff : 0) + e;
            int32_t B;
            double st;
            if (kFirst) {
                const int32_t J = __ldg((ry ? L.col1 : L.col0) + e) + (ry ? L.n : 0);
                B = cur[J];
                st = -__ldg((ry ? L.val1 : L.val0) + e) / sqrt(rd * dcr[J]);
                sbuf[ei] = st;
                bbuf[ei] = B;
            } else {
                B = bbuf[ei];
                st = sbuf[ei];
            }
            if (B != rA && st > 0.0 && (kFirst || mate[B] < 0)) {
                sv = st;
                sj = B;
            }
        }
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
    if (I < rows) {
        cand_s[I] = best_s[w][lane];
        cand_b[I] = act ? best_j[w][lane] : -1;
    }
}

// A node's pick: the best candidate of its member rows (mem, by position).
__global__ void k_nodepick(const int32_t *count, const int32_t *size, const int32_t *mem,
                           const double *cand_s, const int32_t *cand_b, const int32_t *mate,
                           int32_t *pick) {
    pdl_enter();
    const int32_t A = blockIdx.x * blockDim.x + threadIdx.x;
    if (A >= *count) return;
    double best = 0.0;
    int32_t bj = -1;
    if (mate[A] < 0) {
        const int k = size[A];
        for (int p = 0; p < k; ++p) {
            const int32_t m = mem[4 * A + p];
            pick_merge(cand_s[m], cand_b[m], best, bj);
        }
    }
    pick[A] = bj;
}

__global__ void k_handshake(const int32_t *count, const int32_t *pick, int32_t *mate) {
    pdl_enter();
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= *count) return;
    const int32_t J = pick[I];
    if (mate[I] < 0 && J >= 0 && pick[J] == I) mate[I] = J;
}

__global__ void k_leader_flag(const int32_t *count, const int32_t *mate, int32_t *flag) {
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
    const int32_t n = *count;
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] += tile_sum[i / kScanTile];
}

// ---- level bookkeeping --------------------------------------------------------

__global__ void k_number(const int32_t *count, const int32_t *mate, const int32_t *scan,
                         int32_t *cid, const int32_t *size_old, int32_t *size_new) {
    pdl_enter();
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= *count) return;
    const int32_t m = mate[I];
    if (m < 0 || I < m) {
        const int32_t J = scan[I];
        cid[I] = J;
        size_new[J] = size_old[I] + (m >= 0 ? size_old[m] : 0);
    } else {
        cid[I] = scan[m];
    }
}

// The last level: every row to its aggregate and position (in place).
__global__ void k_follow(int32_t rows, int32_t *cur, int32_t *pos, const int32_t *mate,
                         const int32_t *cid, const int32_t *size_old) {
    pdl_enter();
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= rows) return;
    const int32_t a = cur[c];
    const int32_t m = mate[a];
    if (m >= 0 && m < a) pos[c] += size_old[m];
    cur[c] = cid[a];
}

// Levels with a next level: row c moves to its new node J (cur_out) and
// position, is listed as J's member at that position (mem, at most 4 per node
// at the levels that read it), and forms t_c = d_c + (its entries whose
// column lies in J, in storage order) for J's diagonal. J is the row's node a
// and its mate b, so an entry is inside J when its column's node (the column
// itself at level 0, kIdentity) is a or b. One warp per 32 rows walks their
// entries 32 at a time as k_pick does; the matching values are staged in
// shared memory with a ballot mask and each lane adds its own row's in
// storage order.
template <bool kIdentity>
__global__ void __launch_bounds__(32 * kPickWarps) k_follow_t(LevelView L, int32_t rows,
                                                              const int32_t *cur_in,
                                                              int32_t *cur_out, int32_t *pos,
                                                              const int32_t *mate,
                                                              const int32_t *cid,
                                                              const int32_t *size_old,
                                                              int32_t *mem, double *tbuf) {
    pdl_enter();
    __shared__ double sv_s[kPickWarps][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int32_t base = (blockIdx.x * kPickWarps + w) * 32;
    if (base >= rows) return;  // whole warp
    const int32_t c = base + lane;
    int32_t a = -1, b = -1, e0 = 0, len = 0;
    bool yax = false;
    double t = 0.0;
    if (c < rows) {
        a = kIdentity ? c : cur_in[c];
        b = mate[a];
        int32_t p = pos[c];
        if (b >= 0 && b < a) p += size_old[b];
        const int32_t J = cid[a];
        cur_out[c] = J;
        pos[c] = p;
        mem[4 * J + p] = c;
        const RowRef r = row_of(L, c);
        e0 = r.e0;
        len = r.e1 - r.e0;
        yax = r.off != 0;
        t = diag_of(L, c);
    }
    int32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t x = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += x;
    }
    const int32_t excl = incl - len;
    const int32_t T = __shfl_sync(0xffffffffu, incl, 31);
    for (int32_t t0 = 0; t0 < T; t0 += 32) {
        const int32_t q = t0 + lane;
        int row = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
            const int cand = row + step;
            const int32_t ex = __shfl_sync(0xffffffffu, excl, cand & 31);
            if (cand < 32 && ex <= q) row = cand;
        }
        const int32_t re0 = __shfl_sync(0xffffffffu, e0, row);
        const int32_t rex = __shfl_sync(0xffffffffu, excl, row);
        const bool ry = __shfl_sync(0xffffffffu, yax, row);
        const int32_t ra = __shfl_sync(0xffffffffu, a, row);
        const int32_t rb = __shfl_sync(0xffffffffu, b, row);
        double v = 0.0;
        bool hit = false;
        if (q < T) {
            const int32_t e = re0 + (q - rex);
            const int32_t col = __ldg((ry ? L.col1 : L.col0) + e) + (ry ? L.n : 0);
            const int32_t node = kIdentity ? col : cur_in[col];
            hit = node == ra || node == rb;
            if (hit) v = __ldg((ry ? L.val1 : L.val0) + e);
        }
        const unsigned hm = __ballot_sync(0xffffffffu, hit);
        sv_s[w][lane] = v;
        __syncwarp();
        // this lane's row occupies chunk positions [lo, hi): its hits, lowest
        // (earliest stored) first
        const int32_t lo = excl > t0 ? excl - t0 : 0;
        const int32_t hi = excl + len < t0 + 32 ? excl + len - t0 : 32;
        unsigned mine = 0u;
        if (hi > lo) mine = hm & ((hi - lo == 32 ? 0xffffffffu : ((1u << (hi - lo)) - 1u)) << lo);
        while (mine) {
            const int k = __ffs(mine) - 1;
            t += sv_s[w][k];
            mine &= mine - 1u;
        }
        __syncwarp();
    }
    if (c < rows) tbuf[c] = t;
}

// Node J of the next level: its diagonal, the members' t in position order,
// given to each member row (dcr), and its mate cleared for the next level's
// matching.
__global__ void k_dc(const int32_t *count, const int32_t *size, const int32_t *mem,
                     const double *tbuf, double *dcr, int32_t *mate) {
    pdl_enter();
    const int32_t J = blockIdx.x * blockDim.x + threadIdx.x;
    if (J >= *count) return;
    const int k = size[J];
    int32_t m[4];
    m[0] = mem[4 * J];
    double d = tbuf[m[0]];
#pragma unroll
    for (int p = 1; p < 4; ++p) {
        if (p < k) {
            m[p] = mem[4 * J + p];
            d += tbuf[m[p]];
        }
    }
    dcr[m[0]] = d;
#pragma unroll
    for (int p = 1; p < 4; ++p)
        if (p < k) dcr[m[p]] = d;
    mate[J] = -1;
}

// ---- final layout, permuted system, block inverses -------------------------

__global__ void k_newpos(int32_t rows, const int32_t *cur, const int32_t *pos,
                         const int32_t *agg_start, int32_t *newpos, int32_t *order) {
    pdl_enter();
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= rows) return;
    const int32_t p = agg_start[cur[c]] + pos[c];
    newpos[c] = p;
    order[p] = c;
}

__global__ void k_plen(LevelView L, int32_t rows, const int32_t *order, int32_t *plen) {
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
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
        r0, n, R, kAllAxes, wb, tilebuf,
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
        for (int32_t **p : {&s->mate, &s->pick, &s->flag, &s->cid, &s->size_a, &s->size_b,
                            &s->cur, &s->cur2, &s->pos, &s->cand_b, &s->order, &s->newpos,
                            &s->meta})
            if ((rc = grow(c, p, rows))) return rc;
        if ((rc = grow(c, &s->mem, 4 * rows))) return rc;
        if ((rc = grow(c, &s->agg_start, rows + 1))) return rc;
        if ((rc = grow(c, &s->prp, rows + 1))) return rc;
        for (double **p : {&s->cand_s, &s->tbuf, &s->dc, &s->pdiag, &s->prhs, &s->px})
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
        if ((rc = grow(c, &s->sbuf, nnz))) return rc;
        if ((rc = grow(c, &s->bbuf, nnz))) return rc;
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

// Launches a set-up kernel on the context's stream as a programmatic
// dependent launch (the kernel starts with pdl_enter), so that its blocks are
// scheduled while the kernel before it drains; failures surface through
// cudaGetLastError at the end of each set-up step.
template <typename... P, typename... A>
void launch(ktg_ctx *c, void (*kernel)(P...), int grid, int block, A &&...args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
    ++c->launches;
}

// Exclusive scan of in[0 .. *count) into out, total into *total.
void scan(ktg_ctx *c, AggState *s, const int32_t *in, int32_t *out, const int32_t *count,
          int64_t upper, int32_t *total) {
    const int tiles = blocks_for(upper, kScanTile);
    launch(c, k_scan_tiles, tiles, 1024, in, out, count, s->tile_sum);
    launch(c, k_scan_sums, 1, 1024, s->tile_sum, count, total);
    launch(c, k_scan_add, blocks_for(upper, kT), kT, out, count, s->tile_sum);
}

}  // namespace

void free_agg(ktg_ctx *c) {
    AggState *s = c->agg;
    if (!s) return;
    for (void *p : {(void *)s->mate, (void *)s->pick, (void *)s->flag, (void *)s->cid,
                    (void *)s->size_a, (void *)s->size_b, (void *)s->cur, (void *)s->cur2,
                    (void *)s->pos, (void *)s->mem, (void *)s->cand_b, (void *)s->cand_s,
                    (void *)s->tbuf, (void *)s->dc, (void *)s->sbuf, (void *)s->bbuf,
                    (void *)s->counts, (void *)s->tile_sum, (void *)s->agg_start,
                    (void *)s->order, (void *)s->newpos, (void *)s->prp, (void *)s->pcol,
                    (void *)s->pval, (void *)s->pval32, (void *)s->pdiag, (void *)s->prhs,
                    (void *)s->px, (void *)s->minv, (void *)s->meta, (void *)s->blk_start,
                    (void *)s->gslice, (void *)s->zaz, (void *)s->zd, (void *)s->coarse_einv,
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
        launch(c, k_init, 1, kT, 0, s->cur, s->pos, s->size_a, s->mate, s->counts);
        s->blk_grid = 0;
        c->agg_ready = true;
        KTG_CUDA(c, cudaGetLastError());
        return KTG_OK;
    }
    LevelView L0{};
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
    const int gP = blocks_for(rows, 32 * kPickWarps);
    launch(c, k_init, gR, kT, R, s->cur, s->pos, s->size_a, s->mate, cnt);
    int32_t *size_old = s->size_a, *size_new = s->size_b;
    int32_t *cur = s->cur, *cur_next = s->cur2;
    // per-entry strengths (and, above level 0, neighbour nodes): y rows at yoff
    const int64_t yoff = c->sys_cap_nnz;
    for (int level = 0; level < kLevels; ++level) {
        const int32_t *count = cnt + level;
        for (int round = 0; round < kRounds; ++round) {
            if (level == 0) {
                if (round == 0)
                    launch(c, k_pick<true>, gP, 32 * kPickWarps, L0, count, s->mate, s->pick,
                           s->sbuf, yoff);
                else
                    launch(c, k_pick<false>, gP, 32 * kPickWarps, L0, count, s->mate, s->pick,
                           s->sbuf, yoff);
            } else {
                if (round == 0)
                    launch(c, k_rowpick<true>, gP, 32 * kPickWarps, L0, R, cur, s->mate, s->dc,
                           s->sbuf, s->bbuf, yoff, s->cand_s, s->cand_b);
                else
                    launch(c, k_rowpick<false>, gP, 32 * kPickWarps, L0, R, cur, s->mate, s->dc,
                           s->sbuf, s->bbuf, yoff, s->cand_s, s->cand_b);
                launch(c, k_nodepick, gR, kT, count, size_old, s->mem, s->cand_s, s->cand_b,
                       s->mate, s->pick);
            }
            launch(c, k_handshake, gR, kT, count, s->pick, s->mate);
        }
        launch(c, k_leader_flag, gR, kT, count, s->mate, s->flag);
        scan(c, s, s->flag, s->flag, count, rows, cnt + level + 1);
        launch(c, k_number, gR, kT, count, s->mate, s->flag, s->cid, size_old, size_new);
        if (level + 1 < kLevels) {
            // rows to the next level's nodes, members and diagonals
            if (level == 0)
                launch(c, k_follow_t<true>, gP, 32 * kPickWarps, L0, R, cur, cur_next, s->pos,
                       s->mate, s->cid, size_old, s->mem, s->tbuf);
            else
                launch(c, k_follow_t<false>, gP, 32 * kPickWarps, L0, R, cur, cur_next, s->pos,
                       s->mate, s->cid, size_old, s->mem, s->tbuf);
            launch(c, k_dc, gR, kT, cnt + level + 1, size_new, s->mem, s->tbuf, s->dc,
                   s->mate);
            std::swap(cur, cur_next);
        } else {
            launch(c, k_follow, gR, kT, R, cur, s->pos, s->mate, s->cid, size_old);
        }
        std::swap(size_old, size_new);
    }
    // size_old now holds the aggregate sizes; cnt[kLevels] the aggregate count
    const int32_t *nagg = cnt + kLevels;
    scan(c, s, size_old, s->agg_start, nagg, rows, cnt + 5);
    launch(c, k_newpos, gR, kT, R, cur, s->pos, s->agg_start, s->newpos, s->order);
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
    launch(c, k_plen, gR, kT, L0, R, s->order, s->prp);
    // prp: exclusive scan of the permuted row lengths (cnt[6] = R), total at prp[R]
    scan(c, s, s->prp, s->prp, cnt + 6, rows, s->prp + R);
    // the coarse vector of the current mode comes with the permuted system
    // (the learned one only when it is ready)
    const int zmode = (c->coarse == 3 && !c->coarse_z_ready) ? 0 : c->coarse;
    launch(c, k_pfill_tiles, blocks_for(rows, 32 * kPfWarps), 32 * kPfWarps, L0, R, s->order,
           s->newpos, s->prp, c->sys[0].rhs, c->sys[1].rhs, s->pcol, s->pval, s->pval32, s->pdiag,
           s->prhs, zmode, c->coarse_head_w, c->coarse_emb, c->coarse_logd, s->zd);
    launch(c, k_blockinv_lanes, blocks_for(rows, kInvPerBlock), 32 * kInvWarps, nagg,
           s->agg_start, s->final_size, static_cast<int32_t>(n), s->prp, s->pcol, s->pval,
           s->pdiag, s->minv, s->meta);
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
        launch(c, k_coarse_z, blocks_for(rows, kT), kT, mode, R, n, s->prp, s->pval, s->pdiag,
               s->order, c->coarse_head_w, c->coarse_emb, c->coarse_logd, s->zd);
        s->z_mode = mode;
        s->z_gen = c->coarse_z_gen;
    }
    // one even wave of 256-thread blocks (6 per SM), at least 256 rows each
    const int64_t slots = 6ll * c->num_sms;
    const int32_t per = static_cast<int32_t>(std::max<int64_t>(256, (rows + slots - 1) / slots));
    const int blocks = static_cast<int>((rows + per - 1) / per);
    if (2 * blocks > 2 * ((rows + kT - 1) / kT))
        return set_error(c, KTG_ERR_STATE, "coarse partials buffer too small");
    launch(c, k_coarse_az, blocks, kAzThreads, s->prp, s->pcol, s->pval, s->pdiag, s->zd, n,
           R, per, s->zaz, s->coarse_part, s->ticket,
           s->coarse_einv);
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
        launch(c, k_blkstart, blocks_for(grid + 1, kT), kT, grid, static_cast<int32_t>(rows),
               s->counts + kLevels, s->agg_start, s->blk_start);
        s->blk_grid = grid;
    }
    *rows_cap = static_cast<int32_t>((rows + grid - 1) / grid + kAggMax);
    if (rows > 0) {
        launch(c, k_perm_in, blocks_for(rows, kT), kT, static_cast<int32_t>(rows),
               static_cast<int32_t>(c->sys_n), s->order, x, y, s->px);
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
