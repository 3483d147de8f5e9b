// Density-bin occupancy and scaled overflow (sm_100a).
//
// Replaces simplPlacer::Impl::getOccupancy and getOverflow (globalPlacer/
// simpl/simpl_placer.cc:277-297) with BinGrid::getBinOf / clampIndex
// (simpl_grid.h:82-90, 125-127).
//
//   k_occ_accum     one thread per movable cell: bin of the cell centre, area
//                   converted to 64-bit fixed point, lanes of a warp that hit
//                   the same bin combined (match.any) and one integer atomic
//                   per bin and warp. Small grids are first accumulated in a
//                   shared-memory copy of the map (privatised) and flushed
//                   once per block. Integer sums are associative, so the map
//                   is identical from run to run whatever the atomic order.
//   k_occ_finalize  one thread per bin: fixed point -> f64 occupancy, the
//                   overflow term max(occ - g * avail, 0), a deterministic
//                   block sum and a last-block final sum; it also clears the
//                   fixed-point map for the next call.
//
// With areas that are multiples of 2^-s (s = the fixed-point shift, chosen
// from the total movable area so no bin can overflow 63 bits) the map equals
// the reference's sequential f64 sums exactly.
#include "ktg_common.cuh"
#include "ktg_context.h"

#include <algorithm>

namespace ktg {
namespace {

constexpr int kOccThreads = 256;
// Grids with at most this many bins are privatised in (dynamic) shared
// memory: 24576 x 8 B = 192 KiB of the 227 KiB a block may use.
constexpr int kSmemBins = 24576;

struct GridArgs {
    double origin_x, origin_y, dx, dy;
    int32_t nx, ny;
    double scale;
};

// BinGrid::clampIndex: clamp(f, 0, n - 1e-9), truncated.
__device__ __forceinline__ int32_t clamp_index(double f, int32_t n) {
    const double hi = static_cast<double>(n) - 1e-9;
    const double c = f < 0.0 ? 0.0 : (hi < f ? hi : f);
    return static_cast<int32_t>(c);
}

__device__ __forceinline__ int32_t bin_of(const GridArgs &g, double x, double y, double w,
                                          double h) {
    // getCentre: pos + 0.5 * size (simpl_placer.cc:277-280)
    const double cx = x + 0.5 * w;
    const double cy = y + 0.5 * h;
    const int32_t ix = clamp_index((cx - g.origin_x) / g.dx, g.nx);
    const int32_t iy = clamp_index((cy - g.origin_y) / g.dy, g.ny);
    return iy * g.nx + ix;
}

// Sums `v` over the lanes of the calling warp that share `key`; returns the
// sum in the lowest such lane (and whether this lane is it).
__device__ __forceinline__ bool warp_combine(int32_t key, unsigned long long &v) {
    const unsigned group = __match_any_sync(0xffffffffu, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(group) - 1;
    unsigned long long total = 0;
    unsigned rest = group;
    while (rest) {
        const int src = __ffs(rest) - 1;
        rest &= rest - 1;
        total += __shfl_sync(group, v, src);
    }
    v = total;
    return lane == leader;
}

template <bool Private>
__global__ void __launch_bounds__(kOccThreads)
    k_occ_accum(const double *__restrict__ x, const double *__restrict__ y,
                const double *__restrict__ w, const double *__restrict__ h,
                const double *__restrict__ area, int32_t n, GridArgs g,
                unsigned long long *__restrict__ occ_fx) {
    extern __shared__ unsigned long long priv[];
    const int32_t bins = g.nx * g.ny;
    if (Private) {
        for (int32_t k = threadIdx.x; k < bins; k += blockDim.x) priv[k] = 0ull;
        __syncthreads();
    }
    for (int32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const int32_t i = base + threadIdx.x;
        int32_t key = -1;
        unsigned long long v = 0ull;
        if (i < n) {
            key = bin_of(g, x[i], y[i], w[i], h[i]);
            v = static_cast<unsigned long long>(__double2ll_rn(area[i] * g.scale));
        }
        const bool leader = warp_combine(key, v);
        if (leader && key >= 0) {
            if (Private)
                atomicAdd(&priv[key], v);
            else
                atomicAdd(&occ_fx[key], v);
        }
    }
    if (Private) {
        __syncthreads();
        for (int32_t k = threadIdx.x; k < bins; k += blockDim.x)
            if (priv[k] != 0ull) atomicAdd(&occ_fx[k], priv[k]);
    }
}

__global__ void __launch_bounds__(kOccThreads)
    k_occ_finalize(unsigned long long *__restrict__ occ_fx, const double *__restrict__ avail,
                   int32_t bins, double inv_scale, double density_limit, double total_avail,
                   double *__restrict__ occ_out, double *__restrict__ partials,
                   unsigned *__restrict__ ticket, double *__restrict__ overflow_out) {
    __shared__ double scratch[40];
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    double term = 0.0;
    if (k < bins) {
        const long long fx = static_cast<long long>(occ_fx[k]);
        occ_fx[k] = 0ull;
        const double o = static_cast<double>(fx) * inv_scale;
        if (occ_out) occ_out[k] = o;
        term = ref_max(o - density_limit * avail[k], 0.0);
    }
    const double bs = block_sum(term, scratch);
    if (threadIdx.x == 0) __stcg(partials + blockIdx.x, bs);
    if (last_block_done(ticket)) {
        const double excess = sum_partials(partials, gridDim.x, scratch);
        if (threadIdx.x == 0) *overflow_out = total_avail > 0.0 ? excess / total_avail : 0.0;
    }
}

}  // namespace

int launch_occupancy(ktg_ctx *c, const double *x, const double *y, double *occ_dev,
                     double *overflow_dev) {
    const int64_t bins = c->nx * c->ny;
    GridArgs g{c->origin_x, c->origin_y, c->dx, c->dy, static_cast<int32_t>(c->nx),
               static_cast<int32_t>(c->ny), c->fx_scale};
    const int32_t n = static_cast<int32_t>(c->n);
    if (n > 0) {
        int blocks = static_cast<int>((n + kOccThreads - 1) / kOccThreads);
        if (bins <= kSmemBins) {
            // Enough blocks to cover the SMs, each privatising the whole map.
            blocks = std::min(blocks, c->num_sms);
            const size_t smem = sizeof(unsigned long long) * static_cast<size_t>(bins);
            if (!(c->attr_bits & kAttrOccupancy)) {  // per device: once per context
                KTG_CUDA(c, cudaFuncSetAttribute(k_occ_accum<true>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 static_cast<int>(sizeof(unsigned long long) *
                                                                  kSmemBins)));
                c->attr_bits |= kAttrOccupancy;
            }
            k_occ_accum<true><<<blocks, kOccThreads, smem, c->stream>>>(
                x, y, c->width, c->height, c->area, n, g, c->occ_fx);
        } else {
            k_occ_accum<false><<<blocks, kOccThreads, 0, c->stream>>>(
                x, y, c->width, c->height, c->area, n, g, c->occ_fx);
        }
        ++c->launches;
    }
    const int fblocks = static_cast<int>((bins + kOccThreads - 1) / kOccThreads);
    k_occ_finalize<<<fblocks, kOccThreads, 0, c->stream>>>(
        c->occ_fx, c->avail, static_cast<int32_t>(bins), 1.0 / c->fx_scale, c->density_limit,
        c->total_avail, occ_dev, c->partials, c->counters + 1, overflow_dev);
    ++c->launches;
    KTG_CUDA(c, cudaGetLastError());
    return KTG_OK;
}

}  // namespace ktg
