// Star-model systems on the GPU (sm_100a).
//
// Replaces LinearSystems::buildStar / buildStarAxis (globalPlacer/simpl/
// simpl_lss.cc:116-201), which SimPL's initial rounds use. Every net of three
// or more pins with a movable pin gets a star variable numbered after the
// movable cells, in net order; a two-pin net is one spring between its pins
// (weight w), a star net one spring between each pin and its star (weight
// w p / (p - 1)). A spring adds w to the diagonal of each movable end, -w
// towards a movable other end and the other end's offset (or fixed position
// plus offset) minus the own offset to the right-hand side.
//
// The x and y systems share pattern, values and diagonal; only the
// right-hand sides differ. Each row is summed in the reference's spring
// order (a cell's nets in ascending order, a star's pins in order), so with
// -fmad=false every entry equals the reference's.
#include <algorithm>
#include <vector>

#include "ktg_common.cuh"
#include "ktg_context.h"

namespace ktg {
namespace {

constexpr int kT = 256;

__global__ void k_star_flags(const int32_t *net_start, const int32_t *net_mov, int32_t N,
                             int32_t *flag) {
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < N) flag[k] = (net_start[k + 1] - net_start[k] >= 3 && net_mov[k] > 0) ? 1 : 0;
}

// Exclusive scan in place over `count` int32 values, by one block (the
// arrays here are a few hundred thousand long and built once per design).
__global__ void __launch_bounds__(1024) k_scan_inplace(int32_t *a, int32_t count, int64_t *total) {
    __shared__ int64_t warp_tot[32];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int per = (count + blockDim.x - 1) / blockDim.x;
    const int b0 = threadIdx.x * per;
    const int b1 = min(b0 + per, count);
    int64_t local = 0;
    for (int b = b0; b < b1; ++b) local += a[b];
    int64_t incl = local;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[threadIdx.x >> 5] = incl;
    __syncthreads();
    if (threadIdx.x < 32) {
        const int64_t w = warp_tot[threadIdx.x];
        int64_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (threadIdx.x >= o) wi += t;
        }
        warp_tot[threadIdx.x] = wi - w;
        if (threadIdx.x == 31) carry = wi;
    }
    __syncthreads();
    int64_t run = warp_tot[threadIdx.x >> 5] + incl - local;
    for (int b = b0; b < b1; ++b) {
        const int64_t v = a[b];
        a[b] = static_cast<int32_t>(run);
        run += v;
    }
    if (threadIdx.x == 0) *total = carry;
}

struct StarArgs {
    const int32_t *net_start;
    const int32_t *pin_cell;
    const int32_t *pin_var;
    const double *off_x;
    const double *off_y;
    const double *fixed_x;
    const double *fixed_y;
    const double *net_weight;
    const int32_t *net_mov;
    const int32_t *pin_start;
    const int2 *pin_ref;
    const int32_t *star_of;   // exclusive scan of the star flags (valid where flagged)
    const int32_t *star_net;  // net of each star
    int32_t n;
    int32_t stars;
};

// Off-diagonal entries per row (rows 0..n-1 movable cells, n.. stars).
__global__ void k_star_count(StarArgs S, int32_t *cnt) {
    const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= S.n + S.stars) return;
    int32_t c = 0;
    if (r < S.n) {
        for (int32_t e = S.pin_start[r]; e < S.pin_start[r + 1]; ++e) {
            const int2 ref = S.pin_ref[e];
            const int32_t s = S.net_start[ref.x];
            const int32_t p = S.net_start[ref.x + 1] - s;
            if (p == 2)
                c += S.pin_var[s + (1 - ref.y)] >= 0 ? 1 : 0;
            else if (p >= 3)
                c += 1;  // the net has a movable pin (this one), so it has a star
        }
    } else {
        c = S.net_mov[S.star_net[r - S.n]];
    }
    cnt[r] = c;
}

__global__ void k_star_fill(StarArgs S, const int32_t *row_ptr, int32_t *col, double *val,
                            double *diag, double *rhs_x, double *rhs_y, int32_t *col_y,
                            double *val_y, double *diag_y) {
    const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= S.n + S.stars) return;
    int32_t slot = row_ptr[r];
    double dg = 0.0, rx = 0.0, ry = 0.0;
    auto put = [&](int32_t cidx, double v) {
        col[slot] = cidx;
        val[slot] = v;
        col_y[slot] = cidx;
        val_y[slot] = v;
        ++slot;
    };
    if (r < S.n) {
        for (int32_t e = S.pin_start[r]; e < S.pin_start[r + 1]; ++e) {
            const int2 ref = S.pin_ref[e];
            const int32_t k = ref.x;
            const int32_t s = S.net_start[k];
            const int32_t p = S.net_start[k + 1] - s;
            const double ox = S.off_x[s + ref.y], oy = S.off_y[s + ref.y];
            if (p == 2) {
                const double w = S.net_weight[k];
                const int32_t o = s + (1 - ref.y);
                const int32_t vo = S.pin_var[o];
                dg += w;
                if (vo >= 0) {
                    put(vo, -w);
                    rx += w * (S.off_x[o] - ox);
                    ry += w * (S.off_y[o] - oy);
                } else {
                    const int32_t cell = S.pin_cell[o];
                    rx += w * ((S.fixed_x[cell] + S.off_x[o]) - ox);
                    ry += w * ((S.fixed_y[cell] + S.off_y[o]) - oy);
                }
            } else if (p >= 3) {
                const double w = S.net_weight[k] * static_cast<double>(p) / static_cast<double>(p - 1);
                dg += w;
                put(S.n + S.star_of[k], -w);
                rx += w * (0.0 - ox);
                ry += w * (0.0 - oy);
            }
        }
    } else {
        const int32_t k = S.star_net[r - S.n];
        const int32_t s = S.net_start[k];
        const int32_t p = S.net_start[k + 1] - s;
        const double w = S.net_weight[k] * static_cast<double>(p) / static_cast<double>(p - 1);
        for (int32_t q = 0; q < p; ++q) {
            const int32_t v = S.pin_var[s + q];
            dg += w;
            if (v >= 0) {
                put(v, -w);
                rx += w * (S.off_x[s + q] - 0.0);
                ry += w * (S.off_y[s + q] - 0.0);
            } else {
                const int32_t cell = S.pin_cell[s + q];
                rx += w * ((S.fixed_x[cell] + S.off_x[s + q]) - 0.0);
                ry += w * ((S.fixed_y[cell] + S.off_y[s + q]) - 0.0);
            }
        }
    }
    const double d = ref_max(dg, 1e-12);
    diag[r] = d;
    diag_y[r] = d;
    rhs_x[r] = rx;
    rhs_y[r] = ry;
}

__global__ void k_star_nets(const int32_t *flag_scan, const int32_t *net_start,
                            const int32_t *net_mov, int32_t N, int32_t *star_net) {
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < N && net_start[k + 1] - net_start[k] >= 3 && net_mov[k] > 0) star_net[flag_scan[k]] = k;
}

__global__ void k_copy_rowptr(const int32_t *a, int32_t *b, int32_t count) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) b[i] = a[i];
}

}  // namespace

int build_star(ktg_ctx *c, int64_t *size_out, int (*reserve)(ktg_ctx *, int64_t, int64_t)) {
    const int32_t N = static_cast<int32_t>(c->N);
    const int32_t n = static_cast<int32_t>(c->n);
    int32_t *flag = nullptr, *star_net = nullptr, *cnt = nullptr;
    int64_t *tot = nullptr;
    auto cleanup = [&]() {
        if (flag) cudaFree(flag);
        if (star_net) cudaFree(star_net);
        if (cnt) cudaFree(cnt);
        if (tot) cudaFree(tot);
    };
#define KTG_SCUDA(call)                                     \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) {                            \
            cleanup();                                      \
            return cuda_check(c, e_, #call);                \
        }                                                   \
    } while (0)
    KTG_SCUDA(cudaMalloc(&flag, sizeof(int32_t) * std::max(N, 1)));
    KTG_SCUDA(cudaMalloc(&tot, sizeof(int64_t) * 2));
    if (N > 0) {
        k_star_flags<<<(N + kT - 1) / kT, kT, 0, c->stream>>>(c->net_start, c->net_mov, N, flag);
        k_scan_inplace<<<1, 1024, 0, c->stream>>>(flag, N, tot);
        c->launches += 2;
    } else {
        KTG_SCUDA(cudaMemsetAsync(tot, 0, sizeof(int64_t), c->stream));
    }
    int64_t stars = 0;
    KTG_SCUDA(cudaMemcpyAsync(&stars, tot, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    KTG_SCUDA(cudaStreamSynchronize(c->stream));
    const int64_t rows = n + stars;
    if (rows > 0x3fffffffll) {
        cleanup();
        return set_error(c, KTG_ERR_RANGE, "star system exceeds 32-bit indices");
    }
    KTG_SCUDA(cudaMalloc(&star_net, sizeof(int32_t) * std::max<int64_t>(stars, 1)));
    KTG_SCUDA(cudaMalloc(&cnt, sizeof(int32_t) * (rows + 1)));
    if (N > 0) {
        k_star_nets<<<(N + kT - 1) / kT, kT, 0, c->stream>>>(flag, c->net_start, c->net_mov, N, star_net);
        ++c->launches;
    }
    StarArgs S{c->net_start, c->pin_cell, c->pin_var, c->off_x,    c->off_y,
               c->fixed_x,   c->fixed_y,  c->net_base, c->net_mov, c->pin_start,
               c->pin_ref,   flag,        star_net,    n,          static_cast<int32_t>(stars)};
    // net_base holds weight / (degree - 1); the star build needs the weight
    // itself, which the upload keeps in net_weight.
    S.net_weight = c->net_weight;
    if (rows > 0) {
        k_star_count<<<static_cast<int>((rows + kT - 1) / kT), kT, 0, c->stream>>>(S, cnt);
        KTG_SCUDA(cudaMemsetAsync(cnt + rows, 0, sizeof(int32_t), c->stream));
        k_scan_inplace<<<1, 1024, 0, c->stream>>>(cnt, static_cast<int32_t>(rows + 1), tot + 1);
        c->launches += 2;
    }
    int64_t nnz = 0;
    KTG_SCUDA(cudaMemcpyAsync(&nnz, tot + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    KTG_SCUDA(cudaStreamSynchronize(c->stream));
    int rc = reserve(c, rows, std::max<int64_t>(nnz, c->cap_nnz));
    if (rc) {
        cleanup();
        return rc;
    }
    AxisSystem &X = c->sys[0], &Y = c->sys[1];
    if (rows > 0) {
        k_copy_rowptr<<<static_cast<int>((rows + 1 + kT - 1) / kT), kT, 0, c->stream>>>(
            cnt, X.row_ptr, static_cast<int32_t>(rows + 1));
        k_copy_rowptr<<<static_cast<int>((rows + 1 + kT - 1) / kT), kT, 0, c->stream>>>(
            cnt, Y.row_ptr, static_cast<int32_t>(rows + 1));
        k_star_fill<<<static_cast<int>((rows + kT - 1) / kT), kT, 0, c->stream>>>(
            S, cnt, X.col, X.val, X.diag, X.rhs, Y.rhs, Y.col, Y.val, Y.diag);
        c->launches += 3;
    }
    KTG_SCUDA(cudaGetLastError());
    KTG_SCUDA(cudaStreamSynchronize(c->stream));
    cleanup();
#undef KTG_SCUDA
    *size_out = rows;
    return KTG_OK;
}

}  // namespace ktg
