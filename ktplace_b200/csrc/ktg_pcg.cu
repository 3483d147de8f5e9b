// Jacobi-preconditioned CG for the x and y systems in one persistent,
// cooperative launch (sm_100a).
//
// Replaces solveBothAxes (globalPlacer/simpl/simpl_lss.cc:203-290) and
// SparseSystem::multiply (simpl_lss.h:49-57). The whole solve -- warm start,
// every iteration, the stopping test -- runs inside one kernel, so there is no
// host round trip per iteration. Each block owns a contiguous slice of the
// combined row space [x rows | y rows]; three grid barriers per iteration
// separate
//   A: Ap = A p (8 lanes per row, coalesced val/col loads) and p.Ap partials
//   B: x += a p, r -= a Ap, z = r / diag, and r.r, r.z partials
//   C: p = z + b p
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

#include <algorithm>

namespace ktg {
namespace {

constexpr int kPcgThreads = 512;
constexpr int kLanesPerRow = 8;

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
};

enum Slot { kBB = 0, kRZ0 = 1, kRR0 = 2, kPAP = 3, kRR = 4, kRZ = 5 };

__device__ __forceinline__ double *slot_ptr(const PcgArgs &A, int slot, int axis) {
    return A.part + (static_cast<size_t>(slot) * 2 + axis) * gridDim.x;
}

// Block-sums `v` (per-thread) and stores the block partial of (slot, axis).
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

// Sums the grid's partials of K (slot, axis) pairs in a fixed order.
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

__global__ void __launch_bounds__(kPcgThreads) k_pcg(PcgArgs A) {
    __shared__ double scratch[33 * 4];
    __shared__ PcgAxis sax[2];
    if (threadIdx.x < 2) sax[threadIdx.x] = A.ax[threadIdx.x];
    __syncthreads();
    const uint64_t t_start = global_timer_ns();
    const uint64_t total_deadline = t_start + A.total_timeout_ns;
    const int32_t n0 = sax[0].n;
    const int32_t r0 = blockIdx.x * A.rows_per_block;
    const int32_t r1 = min(r0 + A.rows_per_block, A.total_rows);
    const int lane = threadIdx.x & 31;
    const int sub = lane & (kLanesPerRow - 1);
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    constexpr int kRowsPerWarp = kWarp / kLanesPerRow;

    auto deadline = [&]() {
        const uint64_t d = global_timer_ns() + A.barrier_timeout_ns;
        return d < total_deadline ? d : total_deadline;
    };

    // ---- start: Ap = A x, r = b - Ap, z = r / diag, p = z ------------------
    {
        double acc[6] = {0, 0, 0, 0, 0, 0};  // bb, rz, rr for x then y
        for (int32_t base = r0 + warp * kRowsPerWarp; base < r1; base += nwarps * kRowsPerWarp) {
            const int32_t c = base + (lane / kLanesPerRow);
            const bool valid = c < r1;
            const int axis = (valid && c >= n0) ? 1 : 0;
            const PcgAxis &S = sax[axis];
            const int32_t i = valid ? c - (axis ? n0 : 0) : 0;
            double s = 0.0;
            if (valid) {
                const int32_t e1 = __ldg(S.rp + i + 1);
                for (int32_t e = __ldg(S.rp + i) + sub; e < e1; e += kLanesPerRow)
                    s += __ldg(S.val + e) * __ldcg(S.x + __ldg(S.col + e));
            }
            s += __shfl_xor_sync(0xffffffffu, s, 4);
            s += __shfl_xor_sync(0xffffffffu, s, 2);
            s += __shfl_xor_sync(0xffffffffu, s, 1);
            if (valid && sub == 0) {
                const double ap = S.diag[i] * S.x[i] + s;
                const double b = S.rhs[i];
                const double r = b - ap;
                const double z = r / S.diag[i];
                S.r[i] = r;
                S.z[i] = z;
                S.p[i] = z;
                acc[axis * 3 + 0] += b * b;
                acc[axis * 3 + 1] += r * z;
                acc[axis * 3 + 2] += r * r;
            }
        }
        double v0[3] = {acc[0], acc[1], acc[2]};
        double v1[3] = {acc[3], acc[4], acc[5]};
        const int sl[3] = {kBB, kRZ0, kRR0};
        const int a0[3] = {0, 0, 0};
        const int a1[3] = {1, 1, 1};
        store_partials<3>(A, v0, sl, a0, scratch);
        store_partials<3>(A, v1, sl, a1, scratch);
    }
    if (!grid_barrier(A.bar_count, A.bar_gen, A.status, deadline())) return;

    double b_norm[2], rho[2], resid[2];
    bool active[2];
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
        const bool live0 = active[0] && resid[0] > A.tol;
        const bool live1 = active[1] && resid[1] > A.tol;
        if (it >= A.max_iter || !(live0 || live1)) break;
        const bool live[2] = {live0, live1};

        // ---- A: Ap = A p, p.Ap ------------------------------------------
        double pap_acc[2] = {0.0, 0.0};
        for (int32_t base = r0 + warp * kRowsPerWarp; base < r1; base += nwarps * kRowsPerWarp) {
            const int32_t c = base + (lane / kLanesPerRow);
            const int axis = (c < r1 && c >= n0) ? 1 : 0;
            const bool valid = c < r1 && live[axis];
            const PcgAxis &S = sax[axis];
            const int32_t i = c - (axis ? n0 : 0);
            double s = 0.0;
            if (valid) {
                const int32_t e1 = __ldg(S.rp + i + 1);
                for (int32_t e = __ldg(S.rp + i) + sub; e < e1; e += kLanesPerRow)
                    s += __ldg(S.val + e) * __ldcg(S.p + __ldg(S.col + e));
            }
            s += __shfl_xor_sync(0xffffffffu, s, 4);
            s += __shfl_xor_sync(0xffffffffu, s, 2);
            s += __shfl_xor_sync(0xffffffffu, s, 1);
            if (valid && sub == 0) {
                const double pi = S.p[i];
                const double ap = S.diag[i] * pi + s;
                S.ap[i] = ap;
                pap_acc[axis] += pi * ap;
            }
        }
        {
            const int sl[2] = {kPAP, kPAP};
            const int ax[2] = {0, 1};
            store_partials<2>(A, pap_acc, sl, ax, scratch);
        }
        if (!grid_barrier(A.bar_count, A.bar_gen, A.status, deadline())) return;

        double alpha[2] = {0.0, 0.0};
        bool ok[2];
        {
            double pap[2];
            const int sl[2] = {kPAP, kPAP};
            const int ax[2] = {0, 1};
            reduce_partials<2>(A, pap, sl, ax, scratch);
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                ok[a] = live[a] && pap[a] > 0.0;
                if (ok[a]) alpha[a] = rho[a] / pap[a];
            }
        }

        // ---- B: x, r, z update, r.r and r.z ------------------------------
        double acc[4] = {0.0, 0.0, 0.0, 0.0};  // rr x, rz x, rr y, rz y
        for (int32_t c = r0 + threadIdx.x; c < r1; c += blockDim.x) {
            const int axis = c >= n0 ? 1 : 0;
            if (!ok[axis]) continue;
            const PcgAxis &S = sax[axis];
            const int32_t i = c - (axis ? n0 : 0);
            const double a = alpha[axis];
            const double pi = S.p[i];
            S.x[i] += a * pi;
            const double r = S.r[i] - a * S.ap[i];
            const double z = r / S.diag[i];
            S.r[i] = r;
            S.z[i] = z;
            acc[axis * 2 + 0] += r * r;
            acc[axis * 2 + 1] += r * z;
        }
        {
            const int sl[4] = {kRR, kRZ, kRR, kRZ};
            const int ax[4] = {0, 0, 1, 1};
            store_partials<4>(A, acc, sl, ax, scratch);
        }
        if (!grid_barrier(A.bar_count, A.bar_gen, A.status, deadline())) return;

        double beta[2] = {0.0, 0.0};
        bool ok2[2] = {false, false};
        double rho_next[2] = {0.0, 0.0};
        {
            double s[4];
            const int sl[4] = {kRR, kRZ, kRR, kRZ};
            const int ax[4] = {0, 0, 1, 1};
            reduce_partials<4>(A, s, sl, ax, scratch);
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                if (!ok[a]) continue;
                resid[a] = sqrt(s[a * 2 + 0]) / b_norm[a];
                rho_next[a] = s[a * 2 + 1];
                ok2[a] = rho_next[a] > 0.0;
                if (ok2[a]) beta[a] = rho_next[a] / rho[a];
            }
        }

        // ---- C: p = z + beta p -------------------------------------------
        for (int32_t c = r0 + threadIdx.x; c < r1; c += blockDim.x) {
            const int axis = c >= n0 ? 1 : 0;
            if (!ok2[axis]) continue;
            const PcgAxis &S = sax[axis];
            const int32_t i = c - (axis ? n0 : 0);
            S.p[i] = S.z[i] + beta[axis] * S.p[i];
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
        if (!grid_barrier(A.bar_count, A.bar_gen, A.status, deadline())) return;
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

}  // namespace

int launch_solve(ktg_ctx *c, double *x, double *y, double tol, int64_t max_iter,
                 ktg_solve_info *info_dev, double *hist_x, double *hist_y, int64_t hist_cap) {
    const int64_t nsys = c->sys_n;
    PcgArgs A;
    for (int a = 0; a < 2; ++a) {
        ktg::AxisSystem &s = c->sys[a];
        A.ax[a] = PcgAxis{s.row_ptr, s.col, s.val, s.diag, s.rhs, a ? y : x,
                          s.r, s.z, s.p, s.ap, static_cast<int32_t>(nsys)};
    }
    A.total_rows = static_cast<int32_t>(2 * nsys);
    static int max_blocks_per_sm = -1;
    if (max_blocks_per_sm < 0) {
        KTG_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&max_blocks_per_sm, k_pcg,
                                                                   kPcgThreads, 0));
        if (max_blocks_per_sm < 1) return set_error(c, KTG_ERR_CUDA, "k_pcg cannot be resident");
    }
    const int64_t coresident = static_cast<int64_t>(max_blocks_per_sm) * c->num_sms;
    const int64_t want = (A.total_rows + 1023) / 1024;
    const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(coresident, want)));
    A.rows_per_block = static_cast<int32_t>((A.total_rows + grid - 1) / grid);
    if (A.rows_per_block == 0) A.rows_per_block = 1;
    if (c->partials_cap < 12 * static_cast<int64_t>(grid))
        return set_error(c, KTG_ERR_STATE, "partials buffer too small");
    A.tol = tol;
    A.max_iter = max_iter;
    A.part = c->partials;
    A.bar_count = c->counters + 2;
    A.bar_gen = c->counters + 3;
    A.status = c->status;
    A.info = info_dev;
    A.hist_x = hist_x;
    A.hist_y = hist_y;
    A.hist_cap = hist_cap;
    A.barrier_timeout_ns = 2000000000ull;   // 2 s for any single barrier
    A.total_timeout_ns = 120000000000ull;   // 120 s for the whole solve
    KTG_CUDA(c, cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
    // A solve that gave up may have left the arrival counter part-way.
    KTG_CUDA(c, cudaMemsetAsync(c->counters + 2, 0, sizeof(unsigned), c->stream));
    void *args[] = {&A};
    KTG_CUDA(c, cudaLaunchCooperativeKernel((void *)k_pcg, dim3(grid), dim3(kPcgThreads), args, 0,
                                            c->stream));
    k_solve_status<<<1, 1, 0, c->stream>>>(c->status, info_dev);
    c->launches += 2;
    KTG_CUDA(c, cudaGetLastError());
    return KTG_OK;
}

}  // namespace ktg
