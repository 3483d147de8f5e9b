// Jacobi-preconditioned CG for the x and y systems in one persistent,
// cooperative launch (sm_100a).
//
// Replaces solveBothAxes (globalPlacer/simpl/simpl_lss.cc:203-290) and
// SparseSystem::multiply (simpl_lss.h:49-57). The whole solve -- warm start,
// every iteration, the stopping test -- runs inside one kernel, so there is no
// host round trip per iteration. Each block owns a contiguous slice of the
// combined row space [x rows | y rows] (one 1024-thread block per SM); in
// the textbook form three grid barriers per iteration separate
//   A: Ap = A p and p.Ap partials
//   B: x += a p, r -= a Ap, z = r / diag, and r.r, r.z partials
//   C: p = z + b p
// and the default form (3) folds C into A, gathering z and updating p and
// A p = A z + b A p there, for two barriers per iteration.
// When a block's rows fit, its slices of x, r, z, p and Ap live in shared
// memory for the whole solve, so phases B and C never leave the SM and only
// the gathered vector is published to global memory. diag is read through
// L1 instead: every KB of shared memory comes out of the L1 that holds the
// SpMV's gathers in flight (a block with 30 KB more shared memory solved
// the 211k system in 8.6 ms instead of 5.8).
// SpMV runs in one of three shapes (option "pcg_lanes"): warp tiles (the
// default: each warp takes a range of the block's rows balanced by
// nonzeros and streams their nonzeros 32 rows at a time with coalesced
// loads, each lane adding its row's products in storage order), one thread
// per row (same row sums, four gathers in flight), or four lanes per row.
// The first two give the same row sums; their solves are bit-identical in
// form 2 and agree to rounding in the others (dot-product partials group
// rows by thread differently).
// Scalars (alpha, beta, residuals, live flags) are recomputed identically by
// every block from the same partials in a fixed order, so all blocks take the
// same branch and the result is identical from run to run.
//
// Semantics kept from the reference: the two axes step in lock-step while
// live (active and residual > tol), the residual is the recursive ||r||/||b||,
// an axis stops on non-positive p.Ap or r.z, an axis with ||b|| == 0 never
// starts. The per-element updates round exactly like the reference's (no FMA:
// the library is built with -fmad=false); only dot-product and row-sum
// summation orders differ.
#include "ktg_common.cuh"
#include "ktg_context.h"
#include "ktg_spmv.cuh"

#include <algorithm>

namespace ktg {
namespace {

constexpr int kPcgThreads = 1024;
// Shared-memory budget for the per-block vector slices.
constexpr int kPcgSmemBytes = 216 * 1024;
constexpr int kVecsPerRow = 5;  // x, r, z, p, A p (diag is read through L1)
constexpr int kCgVecsPerRow = 7;  // the two-barrier form also keeps s

struct PcgAxis {
    const int32_t *rp;
    const int32_t *col;
    const double *val;
    const double *diag;
    const double *rhs;
    double *x;
    double *r;
    double *z;
    double *p;
    double *ap;
    double *s;
    int32_t n;
};

struct PcgArgs {
    PcgAxis ax[2];
    int32_t total_rows;
    int32_t rows_per_block;
    double tol;
    int64_t max_iter;
    double *part;  // [6 slots][2 axes][grid]
    unsigned *bar_count;
    unsigned *bar_gen;
    int *status;
    ktg_solve_info *info;
    double *hist_x;
    double *hist_y;
    int64_t hist_cap;
    uint64_t barrier_timeout_ns;
    uint64_t total_timeout_ns;
    // reference summation order (form 2): products, chunk partials
    double *prod;     // [3][total_rows], row index axis * n + i
    double *cpart;    // [6][nchunk]
    int32_t nchunk;   // ceil(n / kGrain)
    // FP64 pass after a device-mode mixed solve: when this mixed result shows
    // both axes converged and none stalled, the kernel returns at once
    const ktg_mixed_info *gate;
};

// True (in every thread) when the gate says there is nothing left to solve;
// block 0 then reports zero iterations with the mixed solve's residuals.
__device__ __forceinline__ bool gated_off(const PcgArgs &A) {
    if (!A.gate) return false;
    const ktg_mixed_info g = *A.gate;
    if (!(g.status == 0 && g.stalled == 0 && g.resid_x <= A.tol && g.resid_y <= A.tol))
        return false;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ktg_solve_info inf;
        inf.resid_x = g.resid_x;
        inf.resid_y = g.resid_y;
        inf.iters = 0;
        inf.iters_x = 0;
        inf.iters_y = 0;
        inf.status = 0;
        inf.live = 0;
        *A.info = inf;
    }
    return true;
}

enum Slot { kBB = 0, kRZ0 = 1, kRR0 = 2, kPAP = 3, kRR = 4, kRZ = 5 };

__device__ __forceinline__ double *slot_ptr(const PcgArgs &A, int slot, int axis) {
    return A.part + (static_cast<size_t>(slot) * 2 + axis) * gridDim.x;
}

template <int K>
__device__ __forceinline__ void store_partials(const PcgArgs &A, double (&v)[K],
                                               const int (&slot)[K], const int (&axis)[K],
                                               double *scratch) {
    block_sum_k<K>(v, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) __stcg(slot_ptr(A, slot[k], axis[k]) + blockIdx.x, v[k]);
    }
}

template <int K>
__device__ __forceinline__ void reduce_partials(const PcgArgs &A, double (&out)[K],
                                                const int (&slot)[K], const int (&axis)[K],
                                                double *scratch) {
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = 0.0;
    for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < K; ++k) out[k] += __ldcg(slot_ptr(A, slot[k], axis[k]) + b);
    }
    block_sum_k<K>(out, scratch);
}

// ---- dot products in the reference's summation order (form 2) ----------------
//
// getDeterministicSum (simpl_parallel.h:35-51): chunks of kGrain elements,
// each summed left to right from 0.0, then the chunk sums added in order.
// The products are stored by the phase that computes them; after a grid
// barrier one block per (dot, chunk) adds its chunk's products in order
// (staged in shared memory, the next batch loading while thread 0 adds);
// after a second barrier every block adds the chunk sums in order.
constexpr int kGrain = 4096;
constexpr int kStage = 128;  // chunk sums staged per round (fits the block's scratch)
constexpr int kStageSum = 1024;  // products staged per round (one per thread)

__device__ __forceinline__ double *prod_ptr(const PcgArgs &A, int vec) {
    return A.prod + static_cast<size_t>(vec) * A.total_rows;
}

template <int K>
__device__ bool ref_order_dots(const PcgArgs &A, const int (&vec)[K], const int (&axis)[K],
                               const bool (&want)[K], double (&out)[K], double *sh, double *stage,
                               GridSync &gs, uint64_t deadline_ns) {
    const int32_t n = A.ax[0].n;
    const int32_t nc = A.nchunk;
    const int64_t tasks = static_cast<int64_t>(K) * nc;
    // one block per (dot, chunk): the products are staged kStageSum at a
    // time in shared memory (the next batch already in flight in registers)
    // and thread 0 adds them in index order
    for (int64_t t = blockIdx.x; t < tasks; t += gridDim.x) {
        const int k = static_cast<int>(t / nc), c = static_cast<int>(t % nc);
        bool on = false;
        int v = 0, a = 0;
#pragma unroll
        for (int q = 0; q < K; ++q)
            if (q == k) {
                on = want[q];
                v = vec[q];
                a = axis[q];
            }
        if (!on) continue;
        const double *pr = prod_ptr(A, v) + (a ? n : 0);
        const int32_t b = c * kGrain, e = min(n, b + kGrain);
        double next = static_cast<int32_t>(b + threadIdx.x) < e ? __ldcg(pr + b + threadIdx.x) : 0.0;
        double sum = 0.0;
        for (int32_t base = b; base < e; base += kStageSum) {
            const int32_t cnt = min(kStageSum, e - base);
            __syncthreads();  // the previous batch is consumed
            if (static_cast<int32_t>(threadIdx.x) < cnt) stage[threadIdx.x] = next;
            __syncthreads();
            const int32_t nb = base + kStageSum + static_cast<int32_t>(threadIdx.x);
            next = nb < e ? __ldcg(pr + nb) : 0.0;
            if (threadIdx.x == 0)
                for (int32_t i = 0; i < cnt; ++i) sum += stage[i];
        }
        if (threadIdx.x == 0) __stcg(A.cpart + static_cast<size_t>(k) * nc + c, sum);
    }
    if (!grid_sync(gs, deadline_ns)) return false;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (!want[k]) {
            out[k] = 0.0;
            continue;
        }
        const double *cp = A.cpart + static_cast<size_t>(k) * nc;
        double s = 0.0;
        for (int32_t c0 = 0; c0 < nc; c0 += kStage) {  // staged, then added in order
            const int32_t cnt = min(kStage, nc - c0);
            __syncthreads();
            if (static_cast<int32_t>(threadIdx.x) < cnt) sh[threadIdx.x] = __ldcg(cp + c0 + threadIdx.x);
            __syncthreads();
            if (threadIdx.x == 0)
                for (int32_t c = 0; c < cnt; ++c) s += sh[c];
        }
        __syncthreads();
        if (threadIdx.x == 0) sh[0] = s;
        __syncthreads();
        out[k] = sh[0];
    }
    __syncthreads();
    return true;
}

// Off-diagonal part of row i of S times `in` (gathered from global memory,
// L1 bypassed because other blocks rewrite it between phases), one thread:
// terms are added in storage order, four gathers in flight.
__device__ __forceinline__ double row_offdiag_seq(const PcgAxis &S, int32_t i, double sum,
                                                  const double *in) {
    int32_t e = __ldg(S.rp + i);
    const int32_t e1 = __ldg(S.rp + i + 1);
    for (; e + 4 <= e1; e += 4) {
        const int32_t c0 = __ldg(S.col + e), c1 = __ldg(S.col + e + 1);
        const int32_t c2 = __ldg(S.col + e + 2), c3 = __ldg(S.col + e + 3);
        const double v0 = __ldg(S.val + e), v1 = __ldg(S.val + e + 1);
        const double v2 = __ldg(S.val + e + 2), v3 = __ldg(S.val + e + 3);
        const double g0 = __ldcg(in + c0), g1 = __ldcg(in + c1);
        const double g2 = __ldcg(in + c2), g3 = __ldcg(in + c3);
        sum += v0 * g0;
        sum += v1 * g1;
        sum += v2 * g2;
        sum += v3 * g3;
    }
    for (; e < e1; ++e) sum += __ldg(S.val + e) * __ldcg(in + __ldg(S.col + e));
    return sum;
}

// Same with four lanes per row; every lane of the warp must call it.
__device__ __forceinline__ double row_offdiag_vec4(const PcgAxis &S, int32_t i, bool valid,
                                                   const double *in) {
    const int sub = threadIdx.x & 3;
    double s = 0.0;
    if (valid) {
        int32_t e = __ldg(S.rp + i) + sub;
        const int32_t e1 = __ldg(S.rp + i + 1);
        for (; e + 4 < e1; e += 8) {
            const int32_t c0 = __ldg(S.col + e), c1 = __ldg(S.col + e + 4);
            const double v0 = __ldg(S.val + e), v1 = __ldg(S.val + e + 4);
            const double g0 = __ldcg(in + c0), g1 = __ldcg(in + c1);
            s += v0 * g0;
            s += v1 * g1;
        }
        if (e < e1) s += __ldg(S.val + e) * __ldcg(in + __ldg(S.col + e));
    }
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    return s;
}

constexpr int kTileWarps = kPcgThreads / 32;

// Rec (form 3): A p by the recurrence A p = A z + beta A p_prev, so each
// iteration's SpMV gathers z, published by the update phase before the
// second barrier, and p and A p are updated in the SpMV phase; the third
// barrier (and the phase that published p) goes away. Rounding differs from
// the direct product; iterates agree to rounding.
template <bool Smem, int Lanes, bool Exact = false, bool Rec = false>
__global__ void __launch_bounds__(kPcgThreads, 1) k_pcg(PcgArgs A) {
    if (gated_off(A)) return;
    extern __shared__ __align__(16) double dyn[];
    __shared__ double scratch[33 * 4];
    __shared__ double exstage[Exact ? kStageSum : 1];  // reference-order sums
    __shared__ PcgAxis sax[2];
    if (threadIdx.x < 2) sax[threadIdx.x] = A.ax[threadIdx.x];
    const uint64_t t_start = global_timer_ns();
    const uint64_t total_deadline = t_start + A.total_timeout_ns;
    const int32_t r0 = blockIdx.x * A.rows_per_block;
    const int32_t r1 = min(r0 + A.rows_per_block, A.total_rows);
    const int32_t R = max(r1 - r0, 0);
    const int32_t cap = A.rows_per_block;
    double *sx = dyn, *sr = dyn + cap, *sz = dyn + 2 * cap;
    double *sp = dyn + 3 * cap, *sap = dyn + 4 * cap;
    double *tilebuf = dyn + (Smem ? (kVecsPerRow * cap + 1) / 2 * 2 : 0);  // 16-byte aligned
    __syncthreads();
    const int32_t n0 = sax[0].n;
    auto deadline = [&]() {
        const uint64_t d = global_timer_ns() + A.barrier_timeout_ns;
        return d < total_deadline ? d : total_deadline;
    };
    GridSync gs = grid_sync_init(A.bar_count, A.bar_gen, A.status);
    // warp tiles: per-warp row ranges balanced by nonzeros, fixed for the solve
    __shared__ int32_t wb[kTileWarps + 1];
    if (Lanes == 32) {
        const PcgAxis X = A.ax[0], Y = A.ax[1];
        auto prefix = [&](int32_t c) -> int64_t {  // work of combined rows [0, c)
            const int64_t e = c <= X.n ? int64_t(__ldg(X.rp + c))
                                       : int64_t(__ldg(X.rp + X.n)) + __ldg(Y.rp + (c - X.n));
            return e + int64_t(kRowCost) * c;
        };
        const int32_t rb = min(r0, A.total_rows);  // R == 0 past the last row
        const int64_t base = prefix(rb);
        warp_row_bounds(R, wb, [&](int32_t l) { return prefix(rb + l) - base; });
    }
    // Row l of this block: axis and row index inside that axis.
    auto locate = [&](int32_t l, int &axis, int32_t &i) {
        const int32_t c = r0 + l;
        axis = c >= n0 ? 1 : 0;
        i = c - (axis ? n0 : 0);
    };
    // Vector accessors: shared-memory slice or global array.
#define KTG_V(sm, field) (Smem ? sm[l] : sax[axis].field[i])

    if (Smem) {
        for (int32_t l = threadIdx.x; l < R; l += blockDim.x) {
            int axis;
            int32_t i;
            locate(l, axis, i);
            sx[l] = sax[axis].x[i];
        }
        __syncthreads();
    }

    // SpMV over this block's rows: out[l] = diag * in_own + A_off in_global.
    // `own` reads the row's own input element, `in` selects the gathered
    // vector per axis.
    auto spmv = [&](auto own, auto in_of, auto emit, unsigned live) {
        if (Lanes == 32) {
            double vcur = 0.0;
            warp_tile_spmv<double>(
                r0, n0, R, live, wb, tilebuf,
                [&](int pass, const int32_t *&rp, const int32_t *&col, const double *&val,
                    const double *&in) {
                    rp = sax[pass].rp;
                    col = sax[pass].col;
                    val = sax[pass].val;
                    in = in_of(pass);
                },
                [&](int32_t l, int pass, int32_t i) {
                    const double d = __ldg(sax[pass].diag + i);
                    vcur = own(l, pass, i);
                    return d * vcur;
                },
                [&](int32_t l, int pass, int32_t i, double s) { emit(l, pass, i, vcur, s); });
        } else if (Lanes == 1) {
            for (int32_t l = threadIdx.x; l < R; l += blockDim.x) {
                int axis;
                int32_t i;
                locate(l, axis, i);
                if (!((live >> axis) & 1u)) continue;
                const PcgAxis &S = sax[axis];
                const double d = __ldg(S.diag + i);
                const double v = own(l, axis, i);
                const double s = row_offdiag_seq(S, i, d * v, in_of(axis));
                emit(l, axis, i, v, s);
            }
        } else {
            const int32_t groups = blockDim.x / 4;
            const int32_t g = threadIdx.x / 4;
            for (int32_t base = 0; base < R; base += groups) {
                const int32_t l = base + g;
                int axis = 0;
                int32_t i = 0;
                bool valid = l < R;
                if (valid) locate(l, axis, i);
                if (valid && !((live >> axis) & 1u)) valid = false;
                const PcgAxis &S = sax[axis];
                const double s = row_offdiag_vec4(S, i, valid, in_of(axis));
                if (valid && (threadIdx.x & 3) == 0) {
                    const double d = __ldg(S.diag + i);
                    const double v = own(l, axis, i);
                    emit(l, axis, i, v, d * v + s);
                }
            }
        }
    };

    // ---- start: Ap = A x, r = b - Ap, z = r / diag, p = z ------------------
    {
        double acc[6] = {0, 0, 0, 0, 0, 0};  // bb, rz, rr for x then y
        spmv([&](int32_t l, int axis, int32_t i) { return KTG_V(sx, x); },
             [&](int axis) -> const double * { return sax[axis].x; },
             [&](int32_t l, int axis, int32_t i, double, double ap) {
                 const PcgAxis &S = sax[axis];
                 const double b = __ldg(S.rhs + i);
                 const double r = b - ap;
                 const double d = __ldg(S.diag + i);
                 const double z = r / d;
                 if (Smem) {
                     sr[l] = r;
                     sz[l] = z;
                     sp[l] = z;
                     if (Rec) __stcg(S.z + i, z);
                 } else {
                     S.r[i] = r;
                     S.z[i] = z;
                 }
                 __stcg(S.p + i, z);
                 if constexpr (Exact) {
                     const int32_t ci = axis ? n0 + i : i;
                     __stcg(prod_ptr(A, 0) + ci, b * b);
                     __stcg(prod_ptr(A, 1) + ci, r * z);
                     __stcg(prod_ptr(A, 2) + ci, r * r);
                 } else if (axis) {
                     acc[3] += b * b;
                     acc[4] += r * z;
                     acc[5] += r * r;
                 } else {
                     acc[0] += b * b;
                     acc[1] += r * z;
                     acc[2] += r * r;
                 }
             },
             kAllAxes);
        if constexpr (!Exact) {
            double v0[3] = {acc[0], acc[1], acc[2]};
            double v1[3] = {acc[3], acc[4], acc[5]};
            const int sl[3] = {kBB, kRZ0, kRR0};
            const int a0[3] = {0, 0, 0};
            const int a1[3] = {1, 1, 1};
            store_partials<3>(A, v0, sl, a0, scratch);
            store_partials<3>(A, v1, sl, a1, scratch);
        }
    }
    if (!grid_sync(gs, deadline())) return;

    double b_norm[2], rho[2], resid[2];
    bool active[2];
    int64_t steps[2] = {0, 0};
    if constexpr (Exact) {
        double s[6];
        const int vec[6] = {0, 1, 2, 0, 1, 2};
        const int ax[6] = {0, 0, 0, 1, 1, 1};
        const bool want[6] = {true, true, true, true, true, true};
        if (!ref_order_dots<6>(A, vec, ax, want, s, scratch, exstage, gs, deadline())) return;
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            b_norm[a] = sqrt(s[3 * a]);
            active[a] = b_norm[a] > 0.0;
            rho[a] = active[a] ? s[3 * a + 1] : 0.0;
            resid[a] = active[a] ? sqrt(s[3 * a + 2]) / b_norm[a] : 0.0;
        }
    } else {
        double s[4];
        const int sl[4] = {kBB, kRZ0, kRR0, kBB};
        const int ax[4] = {0, 0, 0, 1};
        reduce_partials<4>(A, s, sl, ax, scratch);
        double t[2];
        const int sl2[2] = {kRZ0, kRR0};
        const int ax2[2] = {1, 1};
        reduce_partials<2>(A, t, sl2, ax2, scratch);
        const double bb[2] = {s[0], s[3]};
        const double rz[2] = {s[1], t[0]};
        const double rr[2] = {s[2], t[1]};
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            b_norm[a] = sqrt(bb[a]);
            active[a] = b_norm[a] > 0.0;
            rho[a] = active[a] ? rz[a] : 0.0;
            resid[a] = active[a] ? sqrt(rr[a]) / b_norm[a] : 0.0;
        }
    }

    int64_t it = 0;
    double beta_rec[2] = {0.0, 0.0};  // Rec: beta of the previous iteration
    bool first_rec[2] = {true, true};
    for (;;) {
        bool live[2];
        live[0] = active[0] && resid[0] > A.tol;
        live[1] = active[1] && resid[1] > A.tol;
        if (it >= A.max_iter || !(live[0] || live[1])) break;

        // ---- A: Ap = A p, p.Ap ------------------------------------------
        double pap_acc[2] = {0.0, 0.0};
        if constexpr (Rec) {
            // w = A z; p = z + beta p, Ap = w + beta Ap (p = z, Ap = w at first)
            spmv([&](int32_t l, int axis, int32_t i) {
                     return Smem ? sz[l] : __ldcg(sax[axis].z + i);
                 },
                 [&](int axis) -> const double * { return sax[axis].z; },
                 [&](int32_t l, int axis, int32_t i, double zi, double w) {
                     // per-axis values by select: no runtime array index, so
                     // they stay in registers
                     double pn = zi, apn = w;
                     if (!(axis ? first_rec[1] : first_rec[0])) {
                         const double be = axis ? beta_rec[1] : beta_rec[0];
                         pn = zi + be * KTG_V(sp, p);
                         apn = w + be * KTG_V(sap, ap);
                     }
                     KTG_V(sp, p) = pn;
                     KTG_V(sap, ap) = apn;
                     if (axis)
                         pap_acc[1] += pn * apn;
                     else
                         pap_acc[0] += pn * apn;
                 },
                 axis_mask(live[0], live[1]));
        } else {
            spmv([&](int32_t l, int axis, int32_t i) {
                     return Smem ? sp[l] : __ldcg(sax[axis].p + i);
                 },
                 [&](int axis) -> const double * { return sax[axis].p; },
                 [&](int32_t l, int axis, int32_t i, double pi, double ap) {
                     if (Smem)
                         sap[l] = ap;
                     else
                         sax[axis].ap[i] = ap;
                     if constexpr (Exact)
                         __stcg(prod_ptr(A, 0) + (axis ? n0 + i : i), pi * ap);
                     else if (axis)
                         pap_acc[1] += pi * ap;
                     else
                         pap_acc[0] += pi * ap;
                 },
                 axis_mask(live[0], live[1]));
        }
        if constexpr (!Exact) {
            const int sl[2] = {kPAP, kPAP};
            const int ax[2] = {0, 1};
            store_partials<2>(A, pap_acc, sl, ax, scratch);
        }
        if (!grid_sync(gs, deadline())) return;

        double alpha[2] = {0.0, 0.0};
        bool ok[2];
        {
            double pap[2];
            if constexpr (Exact) {
                const int vec[2] = {0, 0};
                const int ax[2] = {0, 1};
                const bool want[2] = {live[0], live[1]};
                if (!ref_order_dots<2>(A, vec, ax, want, pap, scratch, exstage, gs, deadline())) return;
            } else {
                const int sl[2] = {kPAP, kPAP};
                const int ax[2] = {0, 1};
                reduce_partials<2>(A, pap, sl, ax, scratch);
            }
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                ok[a] = live[a] && pap[a] > 0.0;
                if (ok[a]) alpha[a] = rho[a] / pap[a];
            }
        }

        // ---- B: x, r, z update, r.r and r.z ------------------------------
        double acc[4] = {0.0, 0.0, 0.0, 0.0};  // rr x, rz x, rr y, rz y
        for (int32_t l = threadIdx.x; l < R; l += blockDim.x) {
            int axis;
            int32_t i;
            locate(l, axis, i);
            if (!(axis ? ok[1] : ok[0])) continue;
            const PcgAxis &S = sax[axis];
            const double a = axis ? alpha[1] : alpha[0];
            const double pi = KTG_V(sp, p);
            const double apv = KTG_V(sap, ap);
            const double d = __ldg(S.diag + i);
            KTG_V(sx, x) += a * pi;
            const double r = KTG_V(sr, r) - a * apv;
            const double z = r / d;
            KTG_V(sr, r) = r;
            KTG_V(sz, z) = z;
            if (Rec && Smem) __stcg(S.z + i, z);  // gathered by the next SpMV
            if constexpr (Exact) {
                const int32_t ci = axis ? n0 + i : i;
                __stcg(prod_ptr(A, 1) + ci, r * r);
                __stcg(prod_ptr(A, 2) + ci, r * z);
            } else if (axis) {
                acc[2] += r * r;
                acc[3] += r * z;
            } else {
                acc[0] += r * r;
                acc[1] += r * z;
            }
        }
        if constexpr (!Exact) {
            const int sl[4] = {kRR, kRZ, kRR, kRZ};
            const int ax[4] = {0, 0, 1, 1};
            store_partials<4>(A, acc, sl, ax, scratch);
        }
        if (!grid_sync(gs, deadline())) return;

        double beta[2] = {0.0, 0.0};
        bool ok2[2] = {false, false};
        double rho_next[2] = {0.0, 0.0};
        {
            double s[4];
            if constexpr (Exact) {
                const int vec[4] = {1, 2, 1, 2};
                const int ax[4] = {0, 0, 1, 1};
                const bool want[4] = {ok[0], ok[0], ok[1], ok[1]};
                if (!ref_order_dots<4>(A, vec, ax, want, s, scratch, exstage, gs, deadline())) return;
            } else {
                const int sl[4] = {kRR, kRZ, kRR, kRZ};
                const int ax[4] = {0, 0, 1, 1};
                reduce_partials<4>(A, s, sl, ax, scratch);
            }
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                if (!ok[a]) continue;
                resid[a] = sqrt(s[a * 2 + 0]) / b_norm[a];
                rho_next[a] = s[a * 2 + 1];
                ok2[a] = rho_next[a] > 0.0;
                if (ok2[a]) beta[a] = rho_next[a] / rho[a];
            }
        }

        // ---- C: p = z + beta p (Rec: done by the next SpMV phase) -----------
        if constexpr (!Rec) {
            for (int32_t l = threadIdx.x; l < R; l += blockDim.x) {
                int axis;
                int32_t i;
                locate(l, axis, i);
                if (!(axis ? ok2[1] : ok2[0])) continue;
                const double pn = KTG_V(sz, z) + (axis ? beta[1] : beta[0]) * KTG_V(sp, p);
                if (Smem) sp[l] = pn;
                __stcg(sax[axis].p + i, pn);
            }
        } else {
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                if (!live[a]) continue;
                beta_rec[a] = beta[a];
                first_rec[a] = false;
            }
        }
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            if (!live[a]) continue;
            ++steps[a];
            if (!ok[a] || !ok2[a]) active[a] = false;
            if (ok2[a]) rho[a] = rho_next[a];
        }
        if (blockIdx.x == 0 && threadIdx.x == 0 && it < A.hist_cap) {
            if (A.hist_x) A.hist_x[it] = resid[0];
            if (A.hist_y) A.hist_y[it] = resid[1];
        }
        ++it;
        if (!Rec && !grid_sync(gs, deadline())) return;
    }
#undef KTG_V

    if (Smem) {
        for (int32_t l = threadIdx.x; l < R; l += blockDim.x) {
            int axis;
            int32_t i;
            locate(l, axis, i);
            sax[axis].x[i] = sx[l];
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ktg_solve_info inf;
        inf.resid_x = resid[0];
        inf.resid_y = resid[1];
        inf.iters = it;
        inf.iters_x = steps[0];
        inf.iters_y = steps[1];
        inf.status = kStatusOk;
        inf.live = ((active[0] && resid[0] > A.tol) ? 1 : 0) |
                   ((active[1] && resid[1] > A.tol) ? 2 : 0);
        *A.info = inf;
    }
}

// Chronopoulos-Gear form of the same Jacobi-PCG: the SpMV runs on z
// (w = A z) and A p is carried by the recurrence s = w + beta s, so r.z, r.r
// and w.z of one iteration need only two grid barriers instead of three, and
// the vector updates fuse into one pass:
//   barrier A -> gamma = r.z, |r|^2: residual, live test, r.z > 0 test
//   SpMV w = A z, delta = w.z       -> barrier B
//   pAp = delta - beta gamma / alpha_prev (= p.Ap in exact arithmetic),
//   pAp > 0 test, alpha; p = z + beta p, s = w + beta s, x += alpha p,
//   r -= alpha s, z = r / diag, partials of the next gamma and |r|^2.
// Every test and counter is applied at the same point of the reference's
// step (simpl_lss.cc:241-262), so iteration counts and observer histories
// match; p and x round exactly as in the reference, r through s.
template <bool Smem, int Lanes>
__global__ void __launch_bounds__(kPcgThreads, 1) k_pcg_cg(PcgArgs A) {
    if (gated_off(A)) return;
    extern __shared__ __align__(16) double dyn[];
    __shared__ double scratch[33 * 4];
    __shared__ PcgAxis sax[2];
    if (threadIdx.x < 2) sax[threadIdx.x] = A.ax[threadIdx.x];
    const uint64_t t_start = global_timer_ns();
    const uint64_t total_deadline = t_start + A.total_timeout_ns;
    const int32_t r0 = blockIdx.x * A.rows_per_block;
    const int32_t r1 = min(r0 + A.rows_per_block, A.total_rows);
    const int32_t R = max(r1 - r0, 0);
    const int32_t cap = A.rows_per_block;
    double *sx = dyn, *sr = dyn + cap, *sz = dyn + 2 * cap, *sp = dyn + 3 * cap;
    double *ss = dyn + 4 * cap, *sw = dyn + 5 * cap, *sd = dyn + 6 * cap;
    double *tilebuf = dyn + (Smem ? (kCgVecsPerRow * cap + 1) / 2 * 2 : 0);  // 16-byte aligned
    __syncthreads();
    const int32_t n0 = sax[0].n;
    auto deadline = [&]() {
        const uint64_t d = global_timer_ns() + A.barrier_timeout_ns;
        return d < total_deadline ? d : total_deadline;
    };
    GridSync gs = grid_sync_init(A.bar_count, A.bar_gen, A.status);
    // warp tiles: per-warp row ranges balanced by nonzeros, fixed for the solve
    __shared__ int32_t wb[kTileWarps + 1];
    if (Lanes == 32) {
        const PcgAxis X = A.ax[0], Y = A.ax[1];
        auto prefix = [&](int32_t c) -> int64_t {  // work of combined rows [0, c)
            const int64_t e = c <= X.n ? int64_t(__ldg(X.rp + c))
                                       : int64_t(__ldg(X.rp + X.n)) + __ldg(Y.rp + (c - X.n));
            return e + int64_t(kRowCost) * c;
        };
        const int32_t rb = min(r0, A.total_rows);  // R == 0 past the last row
        const int64_t base = prefix(rb);
        warp_row_bounds(R, wb, [&](int32_t l) { return prefix(rb + l) - base; });
    }
    auto locate = [&](int32_t l, int &axis, int32_t &i) {
        const int32_t c = r0 + l;
        axis = c >= n0 ? 1 : 0;
        i = c - (axis ? n0 : 0);
    };
    // Global homes when the slices do not fit in shared memory:
    // x -> x, r -> r, z -> z (also the gathered vector), p -> p, s -> s, w -> ap.
#define KTG_V(sm, field) (Smem ? sm[l] : sax[axis].field[i])

    if (Smem) {
        for (int32_t l = threadIdx.x; l < R; l += blockDim.x) {
            int axis;
            int32_t i;
            locate(l, axis, i);
            sx[l] = sax[axis].x[i];
            sd[l] = __ldg(sax[axis].diag + i);
        }
        __syncthreads();
    }

    auto spmv = [&](auto own, auto in_of, auto emit, unsigned live) {
        if (Lanes == 32) {
            double vcur = 0.0;
            warp_tile_spmv<double>(
                r0, n0, R, live, wb, tilebuf,
                [&](int pass, const int32_t *&rp, const int32_t *&col, const double *&val,
                    const double *&in) {
                    rp = sax[pass].rp;
                    col = sax[pass].col;
                    val = sax[pass].val;
                    in = in_of(pass);
                },
                [&](int32_t l, int pass, int32_t i) {
                    const double d = Smem ? sd[l] : __ldg(sax[pass].diag + i);
                    vcur = own(l, pass, i);
                    return d * vcur;
                },
                [&](int32_t l, int pass, int32_t i, double s) { emit(l, pass, i, vcur, s); });
        } else if (Lanes == 1) {
            for (int32_t l = threadIdx.x; l < R; l += blockDim.x) {
                int axis;
                int32_t i;
                locate(l, axis, i);
                if (!((live >> axis) & 1u)) continue;
                const PcgAxis &S = sax[axis];
                const double d = Smem ? sd[l] : __ldg(S.diag + i);
                const double v = own(l, axis, i);
                const double s = row_offdiag_seq(S, i, d * v, in_of(axis));
                emit(l, axis, i, v, s);
            }
        } else {
            const int32_t groups = blockDim.x / 4;
            const int32_t g = threadIdx.x / 4;
            for (int32_t base = 0; base < R; base += groups) {
                const int32_t l = base + g;
                int axis = 0;
                int32_t i = 0;
                bool valid = l < R;
                if (valid) locate(l, axis, i);
                if (valid && !((live >> axis) & 1u)) valid = false;
                const PcgAxis &S = sax[axis];
                const double s = row_offdiag_vec4(S, i, valid, in_of(axis));
                if (valid && (threadIdx.x & 3) == 0) {
                    const double d = Smem ? sd[l] : __ldg(S.diag + i);
                    const double v = own(l, axis, i);
                    emit(l, axis, i, v, d * v + s);
                }
            }
        }
    };

    // ---- start: Ap = A x, r = b - Ap, z = r / diag --------------------------
    {
        double acc[6] = {0, 0, 0, 0, 0, 0};  // bb, rz, rr for x then y
        spmv([&](int32_t l, int axis, int32_t i) { return KTG_V(sx, x); },
             [&](int axis) -> const double * { return sax[axis].x; },
             [&](int32_t l, int axis, int32_t i, double, double ap) {
                 const PcgAxis &S = sax[axis];
                 const double b = __ldg(S.rhs + i);
                 const double r = b - ap;
                 const double d = Smem ? sd[l] : __ldg(S.diag + i);
                 const double z = r / d;
                 if (Smem) {
                     sr[l] = r;
                     sz[l] = z;
                 } else {
                     S.r[i] = r;
                 }
                 __stcg(S.z + i, z);
                 if (axis) {
                     acc[3] += b * b;
                     acc[4] += r * z;
                     acc[5] += r * r;
                 } else {
                     acc[0] += b * b;
                     acc[1] += r * z;
                     acc[2] += r * r;
                 }
             },
             kAllAxes);
        double v0[3] = {acc[0], acc[1], acc[2]};
        double v1[3] = {acc[3], acc[4], acc[5]};
        const int sl[3] = {kBB, kRZ0, kRR0};
        const int a0[3] = {0, 0, 0};
        const int a1[3] = {1, 1, 1};
        store_partials<3>(A, v0, sl, a0, scratch);
        store_partials<3>(A, v1, sl, a1, scratch);
    }
    if (!grid_sync(gs, deadline())) return;

    double b_norm[2], rho[2], rho_prev[2] = {0.0, 0.0}, alpha_prev[2] = {0.0, 0.0}, resid[2];
    bool active[2], first[2] = {true, true}, stepped[2] = {false, false};
    int64_t steps[2] = {0, 0};
    {
        double s[4];
        const int sl[4] = {kBB, kRZ0, kRR0, kBB};
        const int ax[4] = {0, 0, 0, 1};
        reduce_partials<4>(A, s, sl, ax, scratch);
        double t[2];
        const int sl2[2] = {kRZ0, kRR0};
        const int ax2[2] = {1, 1};
        reduce_partials<2>(A, t, sl2, ax2, scratch);
        const double bb[2] = {s[0], s[3]};
        const double rz[2] = {s[1], t[0]};
        const double rr[2] = {s[2], t[1]};
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            b_norm[a] = sqrt(bb[a]);
            active[a] = b_norm[a] > 0.0;
            rho[a] = active[a] ? rz[a] : 0.0;
            resid[a] = active[a] ? sqrt(rr[a]) / b_norm[a] : 0.0;
        }
    }

    int64_t it = 0;
    for (;;) {
        if (it > 0) {
            // ---- after barrier A: results of the previous update ---------
            double s[4];
            const int sl[4] = {kRR, kRZ, kRR, kRZ};
            const int ax[4] = {0, 0, 1, 1};
            reduce_partials<4>(A, s, sl, ax, scratch);
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                if (!stepped[a]) continue;
                resid[a] = sqrt(s[a * 2 + 0]) / b_norm[a];
                const double rz = s[a * 2 + 1];
                if (rz > 0.0) {
                    rho_prev[a] = rho[a];
                    rho[a] = rz;
                } else {
                    active[a] = false;
                }
            }
            if (blockIdx.x == 0 && threadIdx.x == 0 && it - 1 < A.hist_cap) {
                if (A.hist_x) A.hist_x[it - 1] = resid[0];
                if (A.hist_y) A.hist_y[it - 1] = resid[1];
            }
        }
        bool live[2];
        live[0] = active[0] && resid[0] > A.tol;
        live[1] = active[1] && resid[1] > A.tol;
        if (it >= A.max_iter || !(live[0] || live[1])) break;

        // ---- SpMV: w = A z, w.z ---------------------------------------------
        double wz[2] = {0.0, 0.0};
        spmv([&](int32_t l, int axis, int32_t i) {
                 return Smem ? sz[l] : __ldcg(sax[axis].z + i);
             },
             [&](int axis) -> const double * { return sax[axis].z; },
             [&](int32_t l, int axis, int32_t i, double zi, double w) {
                 if (Smem)
                     sw[l] = w;
                 else
                     sax[axis].ap[i] = w;
                 if (axis)
                     wz[1] += w * zi;
                 else
                     wz[0] += w * zi;
             },
             axis_mask(live[0], live[1]));
        {
            const int sl[2] = {kPAP, kPAP};
            const int ax[2] = {0, 1};
            store_partials<2>(A, wz, sl, ax, scratch);
        }
        if (!grid_sync(gs, deadline())) return;

        double alpha[2] = {0.0, 0.0}, beta[2] = {0.0, 0.0};
        bool ok[2];
        {
            double delta[2];
            const int sl[2] = {kPAP, kPAP};
            const int ax[2] = {0, 1};
            reduce_partials<2>(A, delta, sl, ax, scratch);
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                ok[a] = false;
                if (!live[a]) continue;
                double pap = delta[a];
                if (!first[a]) {
                    beta[a] = rho[a] / rho_prev[a];
                    pap = delta[a] - beta[a] * rho[a] / alpha_prev[a];
                }
                ok[a] = pap > 0.0;
                if (ok[a]) alpha[a] = rho[a] / pap;
            }
        }

        // ---- fused update ------------------------------------------------
        double acc[4] = {0.0, 0.0, 0.0, 0.0};  // rr x, rz x, rr y, rz y
        for (int32_t l = threadIdx.x; l < R; l += blockDim.x) {
            int axis;
            int32_t i;
            locate(l, axis, i);
            if (!(axis ? ok[1] : ok[0])) continue;
            const PcgAxis &S = sax[axis];
            const double zi = KTG_V(sz, z);
            const double wi = Smem ? sw[l] : S.ap[i];
            const bool f = axis ? first[1] : first[0];
            const double be = axis ? beta[1] : beta[0];
            const double pn = f ? zi : zi + be * KTG_V(sp, p);
            const double sn = f ? wi : wi + be * KTG_V(ss, s);
            KTG_V(sp, p) = pn;
            KTG_V(ss, s) = sn;
            const double a = axis ? alpha[1] : alpha[0];
            KTG_V(sx, x) += a * pn;
            const double r = KTG_V(sr, r) - a * sn;
            const double d = Smem ? sd[l] : __ldg(S.diag + i);
            const double z = r / d;
            KTG_V(sr, r) = r;
            if (Smem) sz[l] = z;
            __stcg(S.z + i, z);
            if (axis) {
                acc[2] += r * r;
                acc[3] += r * z;
            } else {
                acc[0] += r * r;
                acc[1] += r * z;
            }
        }
        {
            const int sl[4] = {kRR, kRZ, kRR, kRZ};
            const int ax[4] = {0, 0, 1, 1};
            store_partials<4>(A, acc, sl, ax, scratch);
        }
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            stepped[a] = ok[a];
            if (!live[a]) continue;
            ++steps[a];
            if (!ok[a]) {
                active[a] = false;
                continue;
            }
            alpha_prev[a] = alpha[a];
            first[a] = false;
        }
        ++it;
        if (!grid_sync(gs, deadline())) return;
    }
#undef KTG_V

    if (Smem) {
        for (int32_t l = threadIdx.x; l < R; l += blockDim.x) {
            int axis;
            int32_t i;
            locate(l, axis, i);
            sax[axis].x[i] = sx[l];
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ktg_solve_info inf;
        inf.resid_x = resid[0];
        inf.resid_y = resid[1];
        inf.iters = it;
        inf.iters_x = steps[0];
        inf.iters_y = steps[1];
        inf.status = kStatusOk;
        inf.live = ((active[0] && resid[0] > A.tol) ? 1 : 0) |
                   ((active[1] && resid[1] > A.tol) ? 2 : 0);
        *A.info = inf;
    }
}

__global__ void k_solve_status(const int *status, ktg_solve_info *info) {
    if (*status != kStatusOk) info->status = *status;
}

using PcgKernel = void (*)(PcgArgs);

struct Variant {
    PcgKernel fn;
    int vecs_per_row;
};

// form 0: textbook three-barrier PCG; form 1: Chronopoulos-Gear two-barrier;
// form 2: textbook PCG with the reference's summation order everywhere
// (bit-identical to the reference's solve); form 3: textbook PCG with A p by
// recurrence, two barriers.
Variant pick_variant(int form, bool smem, int lanes) {
    if (form == 3) {
        if (lanes == 32)
            return {smem ? k_pcg<true, 32, false, true> : k_pcg<false, 32, false, true>,
                    kVecsPerRow};
        if (smem) return {lanes == 4 ? k_pcg<true, 4, false, true> : k_pcg<true, 1, false, true>,
                          kVecsPerRow};
        return {lanes == 4 ? k_pcg<false, 4, false, true> : k_pcg<false, 1, false, true>,
                kVecsPerRow};
    }
    if (form == 2) {
        if (lanes == 32)
            return {smem ? k_pcg<true, 32, true> : k_pcg<false, 32, true>, kVecsPerRow};
        return {smem ? k_pcg<true, 1, true> : k_pcg<false, 1, true>, kVecsPerRow};
    }
    if (form == 1) {
        if (lanes == 32) return {smem ? k_pcg_cg<true, 32> : k_pcg_cg<false, 32>, kCgVecsPerRow};
        if (smem) return {lanes == 4 ? k_pcg_cg<true, 4> : k_pcg_cg<true, 1>, kCgVecsPerRow};
        return {lanes == 4 ? k_pcg_cg<false, 4> : k_pcg_cg<false, 1>, kCgVecsPerRow};
    }
    if (lanes == 32) return {smem ? k_pcg<true, 32> : k_pcg<false, 32>, kVecsPerRow};
    if (smem) return {lanes == 4 ? k_pcg<true, 4> : k_pcg<true, 1>, kVecsPerRow};
    return {lanes == 4 ? k_pcg<false, 4> : k_pcg<false, 1>, kVecsPerRow};
}

int lanes_index(int lanes) { return lanes == 4 ? 1 : lanes == 32 ? 2 : 0; }

}  // namespace

int pcg_lanes_default = 32;
int pcg_form_default = 3;

int launch_solve(ktg_ctx *c, double *x, double *y, double tol, int64_t max_iter,
                 ktg_solve_info *info_dev, double *hist_x, double *hist_y, int64_t hist_cap) {
    const int64_t nsys = c->sys_n;
    PcgArgs A;
    for (int a = 0; a < 2; ++a) {
        ktg::AxisSystem &s = c->sys[a];
        A.ax[a] = PcgAxis{s.row_ptr, s.col, s.val, s.diag, s.rhs, a ? y : x,
                          s.r, s.z, s.p, s.ap, s.s, static_cast<int32_t>(nsys)};
    }
    A.total_rows = static_cast<int32_t>(2 * nsys);
    // One 1024-thread block per SM; small systems use fewer blocks so each
    // block still owns about a thousand rows.
    const int64_t want = (A.total_rows + 1023) / 1024;
    const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(c->num_sms, want)));
    A.rows_per_block = static_cast<int32_t>((A.total_rows + grid - 1) / grid);
    if (A.rows_per_block == 0) A.rows_per_block = 1;
    const int lanes = c->pcg_lanes > 0 ? c->pcg_lanes : pcg_lanes_default;
    const int form = c->pcg_form >= 0 ? c->pcg_form : pcg_form_default;
    // Dynamic shared memory for the vector slices: what the block may opt in
    // to, less the kernel's static arrays, capped at kPcgSmemBytes.
    size_t &bud = c->pcg_smem_budget[form][lanes_index(lanes)];  // per context (one device)
    if (bud == 0) {
        int optin = 0;
        KTG_CUDA(c, cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                           c->device));
        cudaFuncAttributes fa;
        KTG_CUDA(c, cudaFuncGetAttributes(&fa, pick_variant(form, true, lanes).fn));
        const size_t room = optin > static_cast<int>(fa.sharedSizeBytes)
                                ? static_cast<size_t>(optin) - fa.sharedSizeBytes
                                : 0;
        bud = std::min(room, static_cast<size_t>(kPcgSmemBytes));
        if (bud == 0) bud = 1;
    }
    const int vecs = pick_variant(form, true, lanes).vecs_per_row;
    const size_t tile = lanes == 32 ? sizeof(double) * kTileWarps * kTileChunk : 0;
    const size_t smem =
        sizeof(double) * ((vecs * static_cast<size_t>(A.rows_per_block) + 1) / 2 * 2) + tile;
    const bool use_smem = smem <= bud;
    const Variant v = pick_variant(form, use_smem, lanes);
    const size_t dyn = use_smem ? smem : tile;
    const unsigned bit = 1u << ((form * 2 + (use_smem ? 1 : 0)) * 3 + lanes_index(lanes));
    if (!(c->pcg_attr_bits & bit)) {  // per device: once per context
        KTG_CUDA(c, cudaFuncSetAttribute(v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(bud)));
        c->pcg_attr_bits |= bit;
    }
    int per_sm = 0;
    KTG_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v.fn, kPcgThreads, dyn));
    if (per_sm < 1 || grid > per_sm * c->num_sms)
        return set_error(c, KTG_ERR_CUDA, "PCG blocks cannot all be resident");
    if (c->partials_cap < 12 * static_cast<int64_t>(grid))
        return set_error(c, KTG_ERR_STATE, "partials buffer too small");
    A.tol = tol;
    A.max_iter = max_iter;
    A.part = c->partials;
    A.bar_count = c->counters + 2;
    A.bar_gen = c->counters + 3;
    A.status = c->status;
    A.info = info_dev;
    A.gate = c->pcg_gate;
    A.hist_x = hist_x;
    A.hist_y = hist_y;
    A.hist_cap = hist_cap;
    A.prod = nullptr;
    A.cpart = nullptr;
    A.nchunk = static_cast<int32_t>((nsys + kGrain - 1) / kGrain);
    if (form == 2) {  // products and chunk sums of the reference-order dots
        const int64_t need_prod = 3 * std::max<int64_t>(2 * nsys, 1);
        const int64_t need_cpart = 6 * std::max<int64_t>(A.nchunk, 1);
        if (need_prod > c->exact_prod_cap) {
            if (c->exact_prod) cudaFree(c->exact_prod);
            c->exact_prod = nullptr;
            c->exact_prod_cap = 0;
            KTG_CUDA(c, cudaMalloc(&c->exact_prod, sizeof(double) * need_prod));
            c->exact_prod_cap = need_prod;
        }
        if (need_cpart > c->exact_cpart_cap) {
            if (c->exact_cpart) cudaFree(c->exact_cpart);
            c->exact_cpart = nullptr;
            c->exact_cpart_cap = 0;
            KTG_CUDA(c, cudaMalloc(&c->exact_cpart, sizeof(double) * need_cpart));
            c->exact_cpart_cap = need_cpart;
        }
        A.prod = c->exact_prod;
        A.cpart = c->exact_cpart;
    }
    A.barrier_timeout_ns = 2000000000ull;   // 2 s for any single barrier
    A.total_timeout_ns = 120000000000ull;   // 120 s for the whole solve
    KTG_CUDA(c, cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
    // A solve that gave up may have left the arrival counter part-way.
    KTG_CUDA(c, cudaMemsetAsync(c->counters + 2, 0, sizeof(unsigned), c->stream));
    void *args[] = {&A};
    KTG_CUDA(c, cudaLaunchCooperativeKernel((void *)v.fn, dim3(grid), dim3(kPcgThreads), args,
                                            dyn, c->stream));
    k_solve_status<<<1, 1, 0, c->stream>>>(c->status, info_dev);
    c->launches += 2;
    KTG_CUDA(c, cudaGetLastError());
    return KTG_OK;
}

}  // namespace ktg
