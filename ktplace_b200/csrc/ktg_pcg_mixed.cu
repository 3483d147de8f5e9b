// Mixed-precision Jacobi-PCG with FP64 iterative refinement (sm_100a).
//
// Same systems and stopping rule as solveBothAxes (globalPlacer/simpl/
// simpl_lss.cc:203-290) but the work is split by precision:
//   FP64: the outer residual r = b - A x (FP64 values), the true relative
//         residual ||b - A x|| / ||b|| used as the convergence test, every dot
//         product (accumulated in double) and the alpha/beta scalars;
//   FP32: the CSR values, the inner vectors (d, r, z, p, Ap) and the SpMV
//         inside the correction solve A d = r.
// One persistent cooperative launch runs all refinement rounds of both axes:
//   outer: r = b - A x, test ||r|| / ||b|| <= tol, then solve A d = r in FP32
//          with Jacobi-PCG until ||r_inner|| <= inner_tol * ||r||, x += d.
// A round that fails to halve the true residual is reported as a stall; the
// C ABI then finishes the solve with the FP64 kernel from the current x.
#include "ktg_agg.h"
#include "ktg_common.cuh"
#include "ktg_context.h"
#include "ktg_spmv.cuh"

#include <algorithm>

namespace ktg {
namespace {

constexpr int kMixThreads = 1024;
// An inner solve also stops once its residual is below kFinish * tol * ||b||:
// the round then ends within the tolerance instead of over-solving.
constexpr double kFinish = 0.5;
constexpr int kMixSmemBytes = 216 * 1024;

struct MixAxis {
    const int32_t *rp;
    const int32_t *col;
    const double *val;
    const float *val32;
    const double *diag;
    const double *rhs;
    double *x;
    double *r;    // outer residual (FP64)
    float *d;     // correction
    float *ri;    // inner residual
    float *z;
    float *p;
    float *ap;
    const float *s32;  // learned preconditioner values on A's pattern (null: Jacobi)
    float *rs;         // D^-1/2 r_inner, published for the preconditioner's gathers
    const float *minv;     // aggregation: 8 block-inverse entries per row
    const int32_t *meta;   // aggregation: first row of the aggregate * 8 + size - 1
    int32_t n;
};

struct MixArgs {
    MixAxis ax[2];
    int32_t total_rows;
    int32_t rows_per_block;
    double tol;
    double inner_tol;
    int64_t max_inner;
    int32_t max_outer;
    double *part;  // [8 slots][2 axes][grid]
    unsigned *bar_count;
    unsigned *bar_gen;
    int *status;
    ktg_mixed_info *info;
    double *hist_x;  // true residual after each refinement round
    double *hist_y;
    int64_t hist_cap;
    uint64_t barrier_timeout_ns;
    uint64_t total_timeout_ns;
    const int32_t *blk_start;  // aggregation: block row ranges aligned to aggregates
    double *gslice;            // per-block slices in global memory (null: shared memory)
    // aggregation's coarse correction (null: none): per permuted row (z, (A z)),
    // and per axis 1 / (z^T A z) (0 turns the axis's correction off)
    const float2 *zaz;
    const double *coarse_einv;
    // optional phase timestamps of block 0 (null: none): tag << 56 | %globaltimer
    unsigned long long *trace;
    int32_t trace_cap;
};

enum MixSlot { kTRR = 0, kTBB = 1, kIRZ0 = 2, kIPAP = 3, kIRR = 4, kIRZ = 5, kIZW = 6, kTZR = 7 };

__device__ __forceinline__ double *mslot(const MixArgs &A, int slot, int axis) {
    return A.part + (static_cast<size_t>(slot) * 2 + axis) * gridDim.x;
}

template <int K>
__device__ __forceinline__ void mstore(const MixArgs &A, double (&v)[K], const int (&slot)[K],
                                       const int (&axis)[K], double *scratch) {
    block_sum_k<K>(v, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) __stcg(mslot(A, slot[k], axis[k]) + blockIdx.x, v[k]);
    }
}

template <int K>
__device__ __forceinline__ void mreduce(const MixArgs &A, double (&out)[K], const int (&slot)[K],
                                        const int (&axis)[K], double *scratch) {
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = 0.0;
    for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < K; ++k) out[k] += __ldcg(mslot(A, slot[k], axis[k]) + b);
    }
    block_sum_k<K>(out, scratch);
}

// z_i = r_i / d_i + d_i^-1/2 sum_e s_e rs_j   (M = D^-1/2 (I + S) D^-1/2)
__device__ __forceinline__ float apply_m_row(const MixAxis &S, int32_t i, float r) {
    const float dis = rsqrtf(static_cast<float>(__ldg(S.diag + i)));
    float acc = 0.0f;
    const int32_t e1 = __ldg(S.rp + i + 1);
    for (int32_t e = __ldg(S.rp + i); e < e1; ++e)
        acc += __ldg(S.s32 + e) * __ldcg(S.rs + __ldg(S.col + e));
    return r / static_cast<float>(__ldg(S.diag + i)) + dis * acc;
}

__global__ void __launch_bounds__(kMixThreads, 1) k_pcg_mixed(MixArgs A) {
    __shared__ double scratch[33 * 4];
    __shared__ MixAxis sax[2];
    if (threadIdx.x < 2) sax[threadIdx.x] = A.ax[threadIdx.x];
    __syncthreads();
    const uint64_t total_deadline = global_timer_ns() + A.total_timeout_ns;
    auto deadline = [&]() {
        const uint64_t d = global_timer_ns() + A.barrier_timeout_ns;
        return d < total_deadline ? d : total_deadline;
    };
    const int32_t r0 = blockIdx.x * A.rows_per_block;
    const int32_t r1 = min(r0 + A.rows_per_block, A.total_rows);
    const int32_t n0 = sax[0].n;
    auto locate = [&](int32_t c, int &axis, int32_t &i) {
        axis = c >= n0 ? 1 : 0;
        i = c - (axis ? n0 : 0);
    };
    GridSync gs = grid_sync_init(A.bar_count, A.bar_gen, A.status);
    auto sync = [&]() { return grid_sync(gs, deadline()); };

    double b_norm[2] = {0.0, 0.0}, true_resid[2] = {0.0, 0.0}, prev_resid[2] = {0.0, 0.0};
    bool active[2] = {false, false}, stalled[2] = {false, false};
    int32_t outer[2] = {0, 0};
    int64_t inner[2] = {0, 0};

    for (int round = 0;; ++round) {
        // ---- FP64 residual r = b - A x -------------------------------------
        {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};  // rr x, bb x, rr y, bb y
            for (int32_t c = r0 + threadIdx.x; c < r1; c += blockDim.x) {
                int axis;
                int32_t i;
                locate(c, axis, i);
                const MixAxis &S = sax[axis];
                double s = __ldg(S.diag + i) * __ldcg(S.x + i);
                const int32_t e1 = __ldg(S.rp + i + 1);
                for (int32_t e = __ldg(S.rp + i); e < e1; ++e)
                    s += __ldg(S.val + e) * __ldcg(S.x + __ldg(S.col + e));
                const double b = __ldg(S.rhs + i);
                const double r = b - s;
                S.r[i] = r;
                acc[axis * 2 + 0] += r * r;
                acc[axis * 2 + 1] += b * b;
            }
            const int sl[4] = {kTRR, kTBB, kTRR, kTBB};
            const int ax[4] = {0, 0, 1, 1};
            mstore<4>(A, acc, sl, ax, scratch);
        }
        if (!sync()) return;
        bool live[2];
        double r_norm[2];
        {
            double s[4];
            const int sl[4] = {kTRR, kTBB, kTRR, kTBB};
            const int ax[4] = {0, 0, 1, 1};
            mreduce<4>(A, s, sl, ax, scratch);
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                if (round == 0) {
                    b_norm[a] = sqrt(s[a * 2 + 1]);
                    active[a] = b_norm[a] > 0.0;
                }
                r_norm[a] = sqrt(s[a * 2 + 0]);
                if (active[a]) {
                    prev_resid[a] = true_resid[a];
                    true_resid[a] = r_norm[a] / b_norm[a];
                    // a round must at least halve the true residual
                    if (round > 0 && outer[a] > 0 && !(true_resid[a] < 0.5 * prev_resid[a]) &&
                        true_resid[a] > A.tol)
                        stalled[a] = true;
                }
                live[a] = active[a] && !stalled[a] && true_resid[a] > A.tol &&
                          outer[a] < A.max_outer && inner[a] < A.max_inner;
            }
            if (blockIdx.x == 0 && threadIdx.x == 0 && round > 0 && round - 1 < A.hist_cap) {
                if (A.hist_x) A.hist_x[round - 1] = true_resid[0];
                if (A.hist_y) A.hist_y[round - 1] = true_resid[1];
            }
        }
        if (!(live[0] || live[1])) break;

        // ---- inner FP32 Jacobi-PCG on A d = r ---------------------------------
        const bool pre = sax[0].s32 != nullptr;
        if (pre) {
            // publish D^-1/2 r before the preconditioner gathers it
            for (int32_t c = r0 + threadIdx.x; c < r1; c += blockDim.x) {
                int axis;
                int32_t i;
                locate(c, axis, i);
                if (!live[axis]) continue;
                const MixAxis &S = sax[axis];
                const float r = static_cast<float>(S.r[i]);
                S.ri[i] = r;
                S.d[i] = 0.0f;
                __stcg(S.rs + i, r * rsqrtf(static_cast<float>(__ldg(S.diag + i))));
            }
            if (!sync()) return;
        }
        {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};  // rz x, rr x, rz y, rr y
            for (int32_t c = r0 + threadIdx.x; c < r1; c += blockDim.x) {
                int axis;
                int32_t i;
                locate(c, axis, i);
                if (!live[axis]) continue;
                const MixAxis &S = sax[axis];
                const float r = static_cast<float>(S.r[i]);
                const float z = pre ? apply_m_row(S, i, r) : r / static_cast<float>(__ldg(S.diag + i));
                if (!pre) {
                    S.ri[i] = r;
                    S.d[i] = 0.0f;
                }
                S.z[i] = z;
                __stcg(S.p + i, z);
                acc[axis * 2 + 0] += static_cast<double>(r) * static_cast<double>(z);
                acc[axis * 2 + 1] += static_cast<double>(r) * static_cast<double>(r);
            }
            const int sl[4] = {kIRZ0, kIRR, kIRZ0, kIRR};
            const int ax[4] = {0, 0, 1, 1};
            mstore<4>(A, acc, sl, ax, scratch);
        }
        if (!sync()) return;
        double rho[2] = {0.0, 0.0}, in_resid[2] = {0.0, 0.0}, target[2] = {0.0, 0.0};
        bool in_live[2];
        {
            double s[4];
            const int sl[4] = {kIRZ0, kIRR, kIRZ0, kIRR};
            const int ax[4] = {0, 0, 1, 1};
            mreduce<4>(A, s, sl, ax, scratch);
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                rho[a] = s[a * 2 + 0];
                in_resid[a] = sqrt(s[a * 2 + 1]);
                target[a] = fmax(A.inner_tol * r_norm[a], kFinish * A.tol * b_norm[a]);
                in_live[a] = live[a] && rho[a] > 0.0;
            }
        }
        for (;;) {
#pragma unroll
            for (int a = 0; a < 2; ++a)
                in_live[a] = in_live[a] && in_resid[a] > target[a] && inner[a] < A.max_inner;
            if (!(in_live[0] || in_live[1])) break;
            double pap_acc[2] = {0.0, 0.0};
            for (int32_t c = r0 + threadIdx.x; c < r1; c += blockDim.x) {
                int axis;
                int32_t i;
                locate(c, axis, i);
                if (!in_live[axis]) continue;
                const MixAxis &S = sax[axis];
                const float pi = __ldcg(S.p + i);
                float s = static_cast<float>(__ldg(S.diag + i)) * pi;
                int32_t e = __ldg(S.rp + i);
                const int32_t e1 = __ldg(S.rp + i + 1);
                for (; e + 4 <= e1; e += 4) {
                    const int32_t c0 = __ldg(S.col + e), c1 = __ldg(S.col + e + 1);
                    const int32_t c2 = __ldg(S.col + e + 2), c3 = __ldg(S.col + e + 3);
                    const float g0 = __ldcg(S.p + c0), g1 = __ldcg(S.p + c1);
                    const float g2 = __ldcg(S.p + c2), g3 = __ldcg(S.p + c3);
                    s += __ldg(S.val32 + e) * g0;
                    s += __ldg(S.val32 + e + 1) * g1;
                    s += __ldg(S.val32 + e + 2) * g2;
                    s += __ldg(S.val32 + e + 3) * g3;
                }
                for (; e < e1; ++e) s += __ldg(S.val32 + e) * __ldcg(S.p + __ldg(S.col + e));
                S.ap[i] = s;
                pap_acc[axis] += static_cast<double>(pi) * static_cast<double>(s);
            }
            {
                const int sl[2] = {kIPAP, kIPAP};
                const int ax[2] = {0, 1};
                mstore<2>(A, pap_acc, sl, ax, scratch);
            }
            if (!sync()) return;
            bool ok[2];
            float alpha[2] = {0.0f, 0.0f};
            {
                double pap[2];
                const int sl[2] = {kIPAP, kIPAP};
                const int ax[2] = {0, 1};
                mreduce<2>(A, pap, sl, ax, scratch);
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    ok[a] = in_live[a] && pap[a] > 0.0;
                    if (ok[a]) alpha[a] = static_cast<float>(rho[a] / pap[a]);
                }
            }
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            for (int32_t c = r0 + threadIdx.x; c < r1; c += blockDim.x) {
                int axis;
                int32_t i;
                locate(c, axis, i);
                if (!ok[axis]) continue;
                const MixAxis &S = sax[axis];
                const float a = alpha[axis];
                S.d[i] += a * __ldcg(S.p + i);
                const float r = S.ri[i] - a * S.ap[i];
                S.ri[i] = r;
                acc[axis * 2 + 0] += static_cast<double>(r) * static_cast<double>(r);
                if (pre) {
                    __stcg(S.rs + i, r * rsqrtf(static_cast<float>(__ldg(S.diag + i))));
                } else {
                    const float z = r / static_cast<float>(__ldg(S.diag + i));
                    S.z[i] = z;
                    acc[axis * 2 + 1] += static_cast<double>(r) * static_cast<double>(z);
                }
            }
            if (pre) {
                if (!sync()) return;
                for (int32_t c = r0 + threadIdx.x; c < r1; c += blockDim.x) {
                    int axis;
                    int32_t i;
                    locate(c, axis, i);
                    if (!ok[axis]) continue;
                    const MixAxis &S = sax[axis];
                    const float r = S.ri[i];
                    const float z = apply_m_row(S, i, r);
                    S.z[i] = z;
                    acc[axis * 2 + 1] += static_cast<double>(r) * static_cast<double>(z);
                }
            }
            {
                const int sl[4] = {kIRR, kIRZ, kIRR, kIRZ};
                const int ax[4] = {0, 0, 1, 1};
                mstore<4>(A, acc, sl, ax, scratch);
            }
            if (!sync()) return;
            float beta[2] = {0.0f, 0.0f};
            bool ok2[2] = {false, false};
            {
                double s[4];
                const int sl[4] = {kIRR, kIRZ, kIRR, kIRZ};
                const int ax[4] = {0, 0, 1, 1};
                mreduce<4>(A, s, sl, ax, scratch);
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    if (!ok[a]) continue;
                    in_resid[a] = sqrt(s[a * 2 + 0]);
                    const double rn = s[a * 2 + 1];
                    ok2[a] = rn > 0.0;
                    if (ok2[a]) {
                        beta[a] = static_cast<float>(rn / rho[a]);
                        rho[a] = rn;
                    }
                }
            }
            for (int32_t c = r0 + threadIdx.x; c < r1; c += blockDim.x) {
                int axis;
                int32_t i;
                locate(c, axis, i);
                if (!ok2[axis]) continue;
                const MixAxis &S = sax[axis];
                __stcg(S.p + i, S.z[i] + beta[axis] * __ldcg(S.p + i));
            }
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                if (!in_live[a]) continue;
                ++inner[a];
                if (!ok[a] || !ok2[a]) in_live[a] = false;
            }
            if (!sync()) return;
        }
        // ---- x += d ------------------------------------------------------------
        for (int32_t c = r0 + threadIdx.x; c < r1; c += blockDim.x) {
            int axis;
            int32_t i;
            locate(c, axis, i);
            if (!live[axis]) continue;
            const MixAxis &S = sax[axis];
            S.x[i] += static_cast<double>(S.d[i]);
        }
#pragma unroll
        for (int a = 0; a < 2; ++a)
            if (live[a]) ++outer[a];
        if (!sync()) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ktg_mixed_info inf;
        inf.resid_x = true_resid[0];
        inf.resid_y = true_resid[1];
        inf.inner_x = inner[0];
        inf.inner_y = inner[1];
        inf.outer_x = outer[0];
        inf.outer_y = outer[1];
        inf.status = kStatusOk;
        inf.stalled = (stalled[0] ? 1 : 0) | (stalled[1] ? 2 : 0);
        inf.fp64_iters_x = 0;
        inf.fp64_iters_y = 0;
        *A.info = inf;
    }
}

// Preconditioners of the mixed solve.
enum MixPre { kPreJacobi = 0, kPreLearned = 1, kPreAgg = 2 };

// Chronopoulos-Gear form of the mixed solve, with the block's vector slices
// in shared memory (x, diag in FP64; r, u, w, p, s, d in FP32), or in a
// per-block region of global memory when they do not fit. Per inner
// iteration: w = A u (gather u) and the partials of gamma = r.u, delta = w.u
// and |r|^2 -> barrier -> alpha, beta (FP64) -> p = u + beta p,
// s = w + beta s, d += alpha p, r -= alpha s, u = M r -> barrier.
//   Jacobi:  u = r / d, row-local.
//   learned: u = M r gathers D^-1/2 r of other rows, which adds one barrier.
//   aggregation: the system is renumbered so that every aggregate lies in
//     one block's rows; u = (block inverse) r reads the block's own slice
//     after a __syncthreads, with no extra grid barrier.
template <int PRE>
__global__ void __launch_bounds__(kMixThreads, 1) k_pcg_mixed_cg(MixArgs A) {
    extern __shared__ __align__(16) double dyn[];
    __shared__ double scratch[33 * 8];  // block sums of up to 8 values
    __shared__ MixAxis sax[2];
    if (threadIdx.x < 2) sax[threadIdx.x] = A.ax[threadIdx.x];
    __syncthreads();
    const uint64_t total_deadline = global_timer_ns() + A.total_timeout_ns;
    auto deadline = [&]() {
        const uint64_t d = global_timer_ns() + A.barrier_timeout_ns;
        return d < total_deadline ? d : total_deadline;
    };
    int32_t r0, r1;
    if (PRE == kPreAgg) {
        r0 = __ldg(A.blk_start + blockIdx.x);
        r1 = __ldg(A.blk_start + blockIdx.x + 1);
    } else {
        r0 = blockIdx.x * A.rows_per_block;
        r1 = min(r0 + A.rows_per_block, A.total_rows);
    }
    const int32_t R = max(r1 - r0, 0);
    const int32_t cap = A.rows_per_block;
    // coarse correction of the aggregation preconditioner: u = B^-1 r + z c,
    // c = (z^T r) / (z^T A z) per axis
    const bool coarse = PRE == kPreAgg && A.zaz != nullptr;
    const int slice_doubles = coarse ? 5 : 4;
    double *base = A.gslice ? A.gslice + static_cast<size_t>(blockIdx.x) * cap * 5 : dyn;
    // warp-tile buffer after the shared slices (16-byte aligned)
    double *tile64 =
        A.gslice ? dyn : dyn + (slice_doubles * static_cast<size_t>(cap) + 1) / 2 * 2;
    float *tile32 = reinterpret_cast<float *>(tile64);
    double *sx = base;  // diag is read through L1 (shared memory comes out of L1)
    float *sr = reinterpret_cast<float *>(base + cap);
    // su holds the block part B^-1 r of u (what the SpMV gathers); with the
    // coarse correction the full u is su + z c
    float *su = sr + cap, *sw = su + cap, *sp = sw + cap, *ss = sp + cap, *sdd = ss + cap;
    float2 *szaz = reinterpret_cast<float2 *>(sdd + cap);  // (z, A z) per row (coarse only)
    const int32_t n0 = sax[0].n;
    // phase stamps (tags: 0 entry, 1 prologue done, 2 round start, 3 round's
    // residual reduced, 4 SpMV + partials done, 5 scalars reduced, 6
    // iteration done, 7 exit)
    int32_t ntrace = 0;
    auto stamp = [&](unsigned long long tag) {
        if (A.trace && blockIdx.x == 0 && threadIdx.x == 0 && ntrace < A.trace_cap)
            A.trace[ntrace++] = (tag << 56) | (global_timer_ns() & ((1ull << 56) - 1));
    };
    stamp(0);
    auto locate = [&](int32_t l, int &axis, int32_t &i) {
        const int32_t c = r0 + l;
        axis = c >= n0 ? 1 : 0;
        i = c - (axis ? n0 : 0);
    };
    GridSync gs = grid_sync_init(A.bar_count, A.bar_gen, A.status);
    auto sync = [&]() { return grid_sync(gs, deadline()); };
    constexpr bool pre = PRE == kPreLearned;
    // per-warp row ranges of the warp tiles, balanced by nonzeros (the axes'
    // row pointers may start anywhere in a shared column array)
    __shared__ int32_t wb[kMixThreads / 32 + 1];
    {
        const MixAxis X = A.ax[0], Y = A.ax[1];
        const int64_t x0 = __ldg(X.rp), xn = __ldg(X.rp + X.n), y0 = __ldg(Y.rp);
        auto prefix = [&](int32_t c) -> int64_t {  // work of combined rows [0, c)
            const int64_t e = c <= X.n ? int64_t(__ldg(X.rp + c)) - x0
                                       : (xn - x0) + (int64_t(__ldg(Y.rp + (c - X.n))) - y0);
            return e + int64_t(kRowCost) * c;
        };
        const int32_t rb = min(r0, A.total_rows);
        const int64_t basec = prefix(rb);
        warp_row_bounds(R, wb, [&](int32_t l) { return prefix(rb + l) - basec; });
    }
    for (int32_t l = threadIdx.x; l < R; l += blockDim.x) {
        int axis;
        int32_t i;
        locate(l, axis, i);
        sx[l] = sax[axis].x[i];
        if (coarse) szaz[l] = __ldg(A.zaz + r0 + l);
    }
    double einv[2] = {0.0, 0.0};
    if (coarse) {
        einv[0] = __ldg(A.coarse_einv);
        einv[1] = __ldg(A.coarse_einv + 1);
    }
    __syncthreads();

    // u = M r for own rows with the aggregation preconditioner: the block
    // inverse row of each row times r over its aggregate (own slice).
    auto apply_blocks = [&](unsigned live) {
        __syncthreads();
        for (int32_t l = threadIdx.x; l < R; l += blockDim.x) {
            int axis;
            int32_t i;
            locate(l, axis, i);
            if (!((live >> axis) & 1u)) continue;
            const MixAxis &S = sax[axis];
            const int32_t meta = __ldg(S.meta + i);
            const int k = (meta & 7) + 1;
            const int32_t lf = (meta >> 3) + (axis ? n0 : 0) - r0;
            const float4 m0 = __ldg(reinterpret_cast<const float4 *>(S.minv) + 2 * static_cast<size_t>(i));
            const float4 m1 = __ldg(reinterpret_cast<const float4 *>(S.minv) + 2 * static_cast<size_t>(i) + 1);
            const float mm[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
            float u = 0.0f;
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (q < k) u += mm[q] * sr[lf + q];
            su[l] = u;
            __stcg(S.z + i, u);
        }
    };

    // u = M r for own rows (learned M), reading the published D^-1/2 r: the
    // sum over A's pattern runs as warp tiles, adding in the order and with
    // the roundings of apply_m_row.
    auto apply_m = [&](unsigned live) {
        warp_tile_spmv<float>(
            r0, n0, R, live, wb, tile32,
            [&](int pass, const int32_t *&rp, const int32_t *&col, const float *&val,
                const float *&in) {
                rp = sax[pass].rp;
                col = sax[pass].col;
                val = sax[pass].s32;
                in = sax[pass].rs;
            },
            [&](int32_t, int, int32_t) { return 0.0f; },
            [&](int32_t l, int axis, int32_t i, float acc) {
                const MixAxis &S = sax[axis];
                const float d = static_cast<float>(__ldg(S.diag + i));
                const float u = sr[l] / d + rsqrtf(d) * acc;
                su[l] = u;
                __stcg(S.z + i, u);
            });
    };

    double b_norm[2] = {0.0, 0.0}, true_resid[2] = {0.0, 0.0}, prev_resid[2] = {0.0, 0.0};
    bool active[2] = {false, false}, stalled[2] = {false, false};
    int32_t outer[2] = {0, 0};
    int64_t inner[2] = {0, 0};

    stamp(1);
    for (int round = 0;; ++round) {
        stamp(2);
        // ---- FP64 residual r = b - A x; r32, and u (Jacobi) or D^-1/2 r -----
        {
            // rr x, bb x, rr y, bb y, z.r x, z.r y
            double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            warp_tile_spmv<double>(
                r0, n0, R, kAllAxes, wb, tile64,
                [&](int pass, const int32_t *&rp, const int32_t *&col, const double *&val,
                    const double *&in) {
                    rp = sax[pass].rp;
                    col = sax[pass].col;
                    val = sax[pass].val;
                    in = sax[pass].x;
                },
                [&](int32_t l, int pass, int32_t i) { return __ldg(sax[pass].diag + i) * sx[l]; },
                [&](int32_t l, int axis, int32_t i, double s) {
                    const MixAxis &S = sax[axis];
                    const double b = __ldg(S.rhs + i);
                    const double r = b - s;
                    const float rf = static_cast<float>(r);
                    sr[l] = rf;
                    sdd[l] = 0.0f;
                    if (pre) {
                        __stcg(S.rs + i, rf * rsqrtf(static_cast<float>(__ldg(S.diag + i))));
                    } else if (PRE == kPreJacobi) {
                        const float u = rf / static_cast<float>(__ldg(S.diag + i));
                        su[l] = u;
                        __stcg(S.z + i, u);
                    }
                    const double zr = coarse ? static_cast<double>(szaz[l].x) * r : 0.0;
                    if (axis) {  // per-axis sums in registers (no runtime array index)
                        acc[2] += r * r;
                        acc[3] += b * b;
                        acc[5] += zr;
                    } else {
                        acc[0] += r * r;
                        acc[1] += b * b;
                        acc[4] += zr;
                    }
                });
            if (PRE == kPreAgg) apply_blocks(kAllAxes);
            const int sl[6] = {kTRR, kTBB, kTRR, kTBB, kTZR, kTZR};
            const int ax[6] = {0, 0, 1, 1, 0, 1};
            mstore<6>(A, acc, sl, ax, scratch);
        }
        if (!sync()) return;
        bool live[2];
        double r_norm[2];
        // coarse state per axis: z^T r and z^T s by recurrence, and the
        // coefficient c of z in the current u
        double ztr[2] = {0.0, 0.0}, zts[2] = {0.0, 0.0};
        float cu[2] = {0.0f, 0.0f};
        {
            double s[6];
            const int sl[6] = {kTRR, kTBB, kTRR, kTBB, kTZR, kTZR};
            const int ax[6] = {0, 0, 1, 1, 0, 1};
            mreduce<6>(A, s, sl, ax, scratch);
            if (coarse) {
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    ztr[a] = s[4 + a];
                    cu[a] = static_cast<float>(einv[a] * ztr[a]);
                }
            }
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                if (round == 0) {
                    b_norm[a] = sqrt(s[a * 2 + 1]);
                    active[a] = b_norm[a] > 0.0;
                }
                r_norm[a] = sqrt(s[a * 2 + 0]);
                if (active[a]) {
                    prev_resid[a] = true_resid[a];
                    true_resid[a] = r_norm[a] / b_norm[a];
                    if (round > 0 && outer[a] > 0 && !(true_resid[a] < 0.5 * prev_resid[a]) &&
                        true_resid[a] > A.tol)
                        stalled[a] = true;
                }
                live[a] = active[a] && !stalled[a] && true_resid[a] > A.tol &&
                          outer[a] < A.max_outer && inner[a] < A.max_inner;
            }
            if (blockIdx.x == 0 && threadIdx.x == 0 && round > 0 && round - 1 < A.hist_cap) {
                if (A.hist_x) A.hist_x[round - 1] = true_resid[0];
                if (A.hist_y) A.hist_y[round - 1] = true_resid[1];
            }
        }
        if (!(live[0] || live[1])) break;
        if (pre) {
            apply_m(axis_mask(live[0], live[1]));
            if (!sync()) return;
        }
        // ---- inner FP32 PCG (Chronopoulos-Gear) -------------------------------
        bool in_live[2] = {live[0], live[1]}, first[2] = {true, true};
        double gamma_prev[2] = {0.0, 0.0}, alpha_prev[2] = {0.0, 0.0};
        // inner stop: the round's reduction inner_tol, or as soon as the
        // correction is good enough to finish (half the tolerance left over)
        const double target[2] = {fmax(A.inner_tol * r_norm[0], kFinish * A.tol * b_norm[0]),
                                  fmax(A.inner_tol * r_norm[1], kFinish * A.tol * b_norm[1])};
        stamp(3);
        for (;;) {
            // gamma, delta, rr, z.w per axis
            double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            warp_tile_spmv<float>(
                r0, n0, R, axis_mask(in_live[0], in_live[1]), wb, tile32,
                [&](int pass, const int32_t *&rp, const int32_t *&col, const float *&val,
                    const float *&in) {
                    rp = sax[pass].rp;
                    col = sax[pass].col;
                    val = sax[pass].val32;
                    in = sax[pass].z;
                },
                [&](int32_t l, int pass, int32_t i) {
                    return static_cast<float>(__ldg(sax[pass].diag + i)) * su[l];
                },
                [&](int32_t l, int axis, int32_t, float w) {
                    float ui = su[l];
                    double zw = 0.0;
                    if (coarse) {  // A (u_b + z c) = A u_b + (A z) c
                        const float2 za = szaz[l];
                        const float c = axis ? cu[1] : cu[0];
                        ui += za.x * c;
                        w += za.y * c;
                        zw = static_cast<double>(za.x) * w;
                    }
                    sw[l] = w;
                    const float r = sr[l];
                    const double g = static_cast<double>(r) * ui;
                    const double d = static_cast<double>(w) * ui;
                    const double rr = static_cast<double>(r) * r;
                    if (axis) {  // per-axis sums in registers (no runtime array index)
                        acc[4] += g;
                        acc[5] += d;
                        acc[6] += rr;
                        acc[7] += zw;
                    } else {
                        acc[0] += g;
                        acc[1] += d;
                        acc[2] += rr;
                        acc[3] += zw;
                    }
                });
            if (coarse) {  // one block sum for both axes (each value summed as alone)
                const int sl[8] = {kIRZ, kIPAP, kIRR, kIZW, kIRZ, kIPAP, kIRR, kIZW};
                const int ax[8] = {0, 0, 0, 0, 1, 1, 1, 1};
                mstore<8>(A, acc, sl, ax, scratch);
            } else {
                double a6[6] = {acc[0], acc[1], acc[2], acc[4], acc[5], acc[6]};
                const int sl[6] = {kIRZ, kIPAP, kIRR, kIRZ, kIPAP, kIRR};
                const int ax[6] = {0, 0, 0, 1, 1, 1};
                mstore<6>(A, a6, sl, ax, scratch);
            }
            stamp(4);
            if (!sync()) return;
            float alpha[2] = {0.0f, 0.0f}, beta[2] = {0.0f, 0.0f};
            float cu_next[2] = {cu[0], cu[1]};
            bool ok[2] = {false, false};
            {
                double s[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                if (coarse) {
                    const int sl[8] = {kIRZ, kIPAP, kIRR, kIZW, kIRZ, kIPAP, kIRR, kIZW};
                    const int ax[8] = {0, 0, 0, 0, 1, 1, 1, 1};
                    mreduce<8>(A, s, sl, ax, scratch);
                } else {
                    double s6[6];
                    const int sl[6] = {kIRZ, kIPAP, kIRR, kIRZ, kIPAP, kIRR};
                    const int ax[6] = {0, 0, 0, 1, 1, 1};
                    mreduce<6>(A, s6, sl, ax, scratch);
                    s[0] = s6[0], s[1] = s6[1], s[2] = s6[2];
                    s[4] = s6[3], s[5] = s6[4], s[6] = s6[5];
                }
                const double gamma[2] = {s[0], s[4]}, delta[2] = {s[1], s[5]};
                const double rr[2] = {s[2], s[6]}, zw[2] = {s[3], s[7]};
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    if (!in_live[a]) continue;
                    const double res = sqrt(rr[a]);
                    if (!(res > target[a]) || inner[a] >= A.max_inner || !(gamma[a] > 0.0)) {
                        in_live[a] = false;
                        continue;
                    }
                    double b = 0.0, pap = delta[a];
                    if (!first[a]) {
                        b = gamma[a] / gamma_prev[a];
                        pap = delta[a] - b * gamma[a] / alpha_prev[a];
                    }
                    if (!(pap > 0.0)) {
                        in_live[a] = false;
                        continue;
                    }
                    const double al = gamma[a] / pap;
                    ok[a] = true;
                    alpha[a] = static_cast<float>(al);
                    beta[a] = static_cast<float>(b);
                    gamma_prev[a] = gamma[a];
                    alpha_prev[a] = al;
                    if (coarse) {  // s = w + beta s, r -= alpha s, projected on z
                        zts[a] = first[a] ? zw[a] : zw[a] + b * zts[a];
                        ztr[a] -= al * zts[a];
                        cu_next[a] = static_cast<float>(einv[a] * ztr[a]);
                    }
                }
            }
            stamp(5);
            if (!(ok[0] || ok[1])) break;
            for (int32_t l = threadIdx.x; l < R; l += blockDim.x) {
                int axis;
                int32_t i;
                locate(l, axis, i);
                if (!(axis ? ok[1] : ok[0])) continue;
                const MixAxis &S = sax[axis];
                const bool f = axis ? first[1] : first[0];
                const float al = axis ? alpha[1] : alpha[0];
                const float be = axis ? beta[1] : beta[0];
                const float ui = coarse ? su[l] + szaz[l].x * (axis ? cu[1] : cu[0]) : su[l];
                const float pn = f ? ui : ui + be * sp[l];
                const float sn = f ? sw[l] : sw[l] + be * ss[l];
                sp[l] = pn;
                ss[l] = sn;
                sdd[l] += al * pn;
                const float r = sr[l] - al * sn;
                sr[l] = r;
                if (pre) {
                    __stcg(S.rs + i, r * rsqrtf(static_cast<float>(__ldg(S.diag + i))));
                } else if (PRE == kPreJacobi) {
                    const float u = r / static_cast<float>(__ldg(S.diag + i));
                    su[l] = u;
                    __stcg(S.z + i, u);
                }
            }
            if (PRE == kPreAgg) apply_blocks(axis_mask(ok[0], ok[1]));
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                if (!ok[a]) continue;
                ++inner[a];
                first[a] = false;
                cu[a] = cu_next[a];
            }
            if (!sync()) return;
            stamp(6);
            if (pre) {
                apply_m(axis_mask(ok[0], ok[1]));
                if (!sync()) return;
            }
        }
        // ---- x += d, published for the next residual -------------------------
        for (int32_t l = threadIdx.x; l < R; l += blockDim.x) {
            int axis;
            int32_t i;
            locate(l, axis, i);
            if (!(axis ? live[1] : live[0])) continue;
            sx[l] += static_cast<double>(sdd[l]);
            sax[axis].x[i] = sx[l];
        }
#pragma unroll
        for (int a = 0; a < 2; ++a)
            if (live[a]) ++outer[a];
        if (!sync()) return;
    }
    stamp(7);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ktg_mixed_info inf;
        inf.resid_x = true_resid[0];
        inf.resid_y = true_resid[1];
        inf.inner_x = inner[0];
        inf.inner_y = inner[1];
        inf.outer_x = outer[0];
        inf.outer_y = outer[1];
        inf.status = kStatusOk;
        inf.stalled = (stalled[0] ? 1 : 0) | (stalled[1] ? 2 : 0);
        inf.fp64_iters_x = 0;
        inf.fp64_iters_y = 0;
        *A.info = inf;
    }
}

__global__ void k_to_f32(const double *__restrict__ a, float *__restrict__ b, int64_t n) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        b[i] = static_cast<float>(a[i]);
}

__global__ void k_mixed_status(const int *status, ktg_mixed_info *info) {
    if (*status != kStatusOk) info->status = *status;
}

}  // namespace

int launch_solve_mixed(ktg_ctx *c, double *x, double *y, double tol, double inner_tol,
                       int64_t max_inner, int32_t max_outer, ktg_mixed_info *info_dev,
                       double *hist_x, double *hist_y, int64_t hist_cap) {
    const int64_t nsys = c->sys_n;
    const bool agg = c->precond == 2;
    const bool learned = c->precond == 1 && c->precond_ready;
    int rc = KTG_OK;
    if (agg && !c->agg_ready && (rc = prepare_agg(c))) return rc;
    if (!agg && !c->val32_valid) {
        for (int a = 0; a < 2; ++a) {
            int32_t m = 0;
            KTG_CUDA(c, cudaMemcpyAsync(&m, c->sys[a].row_ptr + nsys, sizeof(int32_t),
                                        cudaMemcpyDeviceToHost, c->stream));
            KTG_CUDA(c, cudaStreamSynchronize(c->stream));
            if (m > 0) {
                const int blocks = static_cast<int>(std::min<int64_t>((m + 255) / 256, 4096));
                k_to_f32<<<blocks, 256, 0, c->stream>>>(c->sys[a].val, c->sys[a].val32, m);
                ++c->launches;
            }
        }
        c->val32_valid = true;
    }
    MixArgs A;
    A.total_rows = static_cast<int32_t>(2 * nsys);
    const int64_t want = (A.total_rows + 1023) / 1024;
    const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(c->num_sms, want)));
    A.rows_per_block = static_cast<int32_t>((A.total_rows + grid - 1) / grid);
    if (A.rows_per_block == 0) A.rows_per_block = 1;
    A.blk_start = nullptr;
    A.gslice = nullptr;
    A.zaz = nullptr;
    A.coarse_einv = nullptr;
    A.trace = c->mixed_trace;
    A.trace_cap = c->mixed_trace_cap;
    AggState *g = nullptr;
    if (agg) {
        if ((rc = agg_prepare_solve(c, grid, x, y, &A.rows_per_block))) return rc;
        g = c->agg;
        A.blk_start = g->blk_start;
        if (c->coarse > 0) {
            if (c->coarse == 3 && !c->coarse_z_ready)
                return set_error(c, KTG_ERR_STATE, "learned coarse vector not prepared");
            if ((rc = agg_coarse_setup(c, c->coarse))) return rc;
            A.zaz = g->zaz;
            A.coarse_einv = g->coarse_einv;
        }
    }
    for (int a = 0; a < 2; ++a) {
        ktg::AxisSystem &s = c->sys[a];
        if (agg) {
            const int64_t o = a * nsys;
            A.ax[a] = MixAxis{g->prp + o, g->pcol, g->pval, g->pval32, g->pdiag + o, g->prhs + o,
                              g->px + o, s.r, s.d32, s.r32, s.z32, s.p32, s.ap32, nullptr,
                              s.rs32, g->minv + o * 8, g->meta + o, static_cast<int32_t>(nsys)};
        } else {
            A.ax[a] = MixAxis{s.row_ptr, s.col, s.val, s.val32, s.diag, s.rhs, a ? y : x, s.r,
                              s.d32, s.r32, s.z32, s.p32, s.ap32, learned ? s.s32 : nullptr,
                              s.rs32, nullptr, nullptr, static_cast<int32_t>(nsys)};
        }
    }
    // Chronopoulos-Gear kernel (always for the aggregation preconditioner),
    // with shared-memory slices of 32 bytes per row when they fit, else
    // global ones; the textbook kernel on global vectors when asked for.
    // 32 bytes per row (x; r, u, w, p, s, d), 40 with the coarse (z, A z)
    const size_t slice = (A.zaz ? 40 : 32) * static_cast<size_t>(A.rows_per_block) + 8;
    const size_t tile = sizeof(double) * kTileChunk * (kMixThreads / 32);
    const bool cg_form = agg || c->mixed_form != 0;
    const bool in_smem = slice + tile <= kMixSmemBytes;
    if (cg_form && !in_smem) {
        A.gslice = agg_global_slices(c, static_cast<int64_t>(grid) * A.rows_per_block * 5);
        if (!A.gslice) return KTG_ERR_NOMEM;
    }
    void (*fn)(MixArgs) = !cg_form ? k_pcg_mixed
                          : agg    ? k_pcg_mixed_cg<kPreAgg>
                          : learned ? k_pcg_mixed_cg<kPreLearned>
                                    : k_pcg_mixed_cg<kPreJacobi>;
    const size_t dyn = !cg_form ? 0 : in_smem ? slice + tile : tile;
    if (!(c->attr_bits & kAttrMixed)) {  // per device: once per context
        for (void (*f)(MixArgs) : {k_pcg_mixed_cg<kPreJacobi>, k_pcg_mixed_cg<kPreLearned>,
                                   k_pcg_mixed_cg<kPreAgg>})
            KTG_CUDA(c, cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             kMixSmemBytes));
        c->attr_bits |= kAttrMixed;
    }
    int per_sm = 0;
    KTG_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kMixThreads, dyn));
    if (per_sm < 1 || grid > per_sm * c->num_sms)
        return set_error(c, KTG_ERR_CUDA, "mixed PCG blocks cannot all be resident");
    if (c->partials_cap < 12 * static_cast<int64_t>(grid))
        return set_error(c, KTG_ERR_STATE, "partials buffer too small");
    A.tol = tol;
    A.inner_tol = inner_tol;
    A.max_inner = max_inner;
    A.max_outer = max_outer;
    A.part = c->partials;
    A.bar_count = c->counters + 2;
    A.bar_gen = c->counters + 3;
    A.status = c->status;
    A.info = info_dev;
    A.hist_x = hist_x;
    A.hist_y = hist_y;
    A.hist_cap = hist_cap;
    A.barrier_timeout_ns = 2000000000ull;
    A.total_timeout_ns = 120000000000ull;
    KTG_CUDA(c, cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
    KTG_CUDA(c, cudaMemsetAsync(c->counters + 2, 0, sizeof(unsigned), c->stream));
    void *args[] = {&A};
    KTG_CUDA(c, cudaLaunchCooperativeKernel((void *)fn, dim3(grid), dim3(kMixThreads), args, dyn,
                                            c->stream));
    k_mixed_status<<<1, 1, 0, c->stream>>>(c->status, info_dev);
    c->launches += 2;
    KTG_CUDA(c, cudaGetLastError());
    if (agg && (rc = agg_finish_solve(c, x, y))) return rc;
    return KTG_OK;
}

}  // namespace ktg
