// Look-ahead legalization on the GPU (sm_100a).
//
// Replaces LookAheadLegalizer::legalize (globalPlacer/simpl/simpl_lal.cc:
// 43-372) with the BinGrid / FreeSpace / AxisProfile arithmetic of
// globalPlacer/simpl/simpl_grid.h, bit for bit:
//
//   host   the cluster loop, which is sequential in the reference: bins of
//          the cell centres and their occupancy (ktg's fixed-point occupancy
//          kernel, exact for the integer site areas of row-based designs),
//          overfilled clusters (4-neighbour flood fill from the lowest bin),
//          growth by the least dense of four one-bin extensions, batches of
//          regions whose one-bin reaches do not touch -- all with the
//          reference's summation order over the host copy of the grid;
//   device each batch: the regions' cells, then the recursive bisection
//          level by level over every block of the batch at once:
//            * cells sorted by (centre, index)          (segmented sort)
//            * per block, in the reference's order on one thread: cell
//              area, the area median m, the free-space profile of the box
//              (vertical: row spans as (x, +-h) steps, segmented sort,
//              running sums), the cutline and the two half boxes;
//            * per half on one thread: its profile, the stripes (obstacle
//              edges, unique, midpoint splits above stripeAreaFraction of
//              the region's room) in the reference's distance-from-cut order;
//            * cells sorted by (-distance from the cut, index), stripes
//              filled greedily in that order (one thread per half);
//            * per stripe the lowest / highest centre (exact atomics on
//              order-preserving bits), then every cell's new position;
//            * children: the low and high cells, next axis.
//          then the bins and occupancy of all cells again for the host.
//
// The sorts are key-only over 16-byte keys: (order bits of a double, index)
// for cells and (order bits of x, order bits of dh) for profile steps; a
// segment of up to kSortSmall keys is sorted by one block in shared memory,
// a longer one by sorted chunks and merge passes.
#include "ktg_common.cuh"
#include "ktg_context.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <vector>

namespace ktg {

namespace {

constexpr int kT = 256;
constexpr int kSortSmall = 2048;

struct Key {
    unsigned long long a, b;
};

__host__ __device__ __forceinline__ bool key_lt(const Key &x, const Key &y) {
    return x.a < y.a || (x.a == y.a && x.b < y.b);
}

// Order-preserving bits of a double; -0.0 counts as +0.0 (the reference's
// comparisons treat them as equal).
__device__ __forceinline__ unsigned long long ord(double v) {
    const unsigned long long u = static_cast<unsigned long long>(__double_as_longlong(v + 0.0));
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

__device__ __forceinline__ double unord(unsigned long long u) {
    const unsigned long long r = (u >> 63) ? (u & 0x7fffffffffffffffull) : ~u;
    return __longlong_as_double(static_cast<long long>(r));
}

// ---- segmented key sort ---------------------------------------------------------

// One block per segment of at most kSortSmall keys: bitonic sort in shared memory.
__global__ void __launch_bounds__(kT) k_sort_small(Key *keys, const int64_t *seg, int nseg) {
    __shared__ Key s[kSortSmall];
    const int sidx = blockIdx.x;
    if (sidx >= nseg) return;
    const int64_t b = seg[2 * sidx], e = seg[2 * sidx + 1];
    const int len = static_cast<int>(e - b);
    int P = 1;
    while (P < len) P <<= 1;
    for (int i = threadIdx.x; i < P; i += kT)
        s[i] = i < len ? keys[b + i] : Key{~0ull, ~0ull};
    __syncthreads();
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += kT) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const Key x = s[i], y = s[ixj];
                    if (key_lt(y, x) == ((i & k) == 0)) {
                        s[i] = y;
                        s[ixj] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < len; i += kT) keys[b + i] = s[i];
}

// Chunks of kSortSmall keys of one long segment, each sorted in shared memory.
__global__ void __launch_bounds__(kT) k_sort_chunks(Key *keys, int64_t b, int64_t e) {
    __shared__ Key s[kSortSmall];
    const int64_t c0 = b + static_cast<int64_t>(blockIdx.x) * kSortSmall;
    const int len = static_cast<int>(std::min<int64_t>(kSortSmall, e - c0));
    for (int i = threadIdx.x; i < kSortSmall; i += kT)
        s[i] = i < len ? keys[c0 + i] : Key{~0ull, ~0ull};
    __syncthreads();
    for (int k = 2; k <= kSortSmall; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < kSortSmall; i += kT) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const Key x = s[i], y = s[ixj];
                    if (key_lt(y, x) == ((i & k) == 0)) {
                        s[i] = y;
                        s[ixj] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < len; i += kT) keys[c0 + i] = s[i];
}

// One merge pass over a long segment: runs of `run` keys pairwise, stable
// (keys of the first run go before equal keys of the second).
__global__ void k_merge_pass(const Key *src, Key *dst, int64_t b, int64_t e, int64_t run) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t len = e - b;
    if (r >= len) return;
    const int64_t pair = r / (2 * run);
    const int64_t a0 = pair * 2 * run;
    const int64_t a1 = std::min(a0 + run, len);
    const int64_t b1 = std::min(a0 + 2 * run, len);
    const Key k = src[b + r];
    int64_t out;
    if (r < a1) {  // in the first run: count second-run keys strictly below
        int64_t lo = a1, hi = b1;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (key_lt(src[b + mid], k)) lo = mid + 1;
            else hi = mid;
        }
        out = a0 + (r - a0) + (lo - a1);
    } else {  // in the second run: count first-run keys not above
        int64_t lo = a0, hi = a1;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (!key_lt(k, src[b + mid])) lo = mid + 1;
            else hi = mid;
        }
        out = a0 + (r - a1) + (lo - a0);
    }
    dst[b + out] = k;
}

__global__ void k_copy_keys(const Key *src, Key *dst, int64_t b, int64_t e) {
    const int64_t i = b + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < e) dst[i] = src[i];
}

int blocks_for(int64_t items, int threads = kT) {
    return static_cast<int>(std::max<int64_t>(1, (items + threads - 1) / threads));
}

// Sorts keys[b, e) of every segment (host list, device copy in dseg).
int seg_sort(ktg_ctx *c, Key *keys, Key *tmp, const std::vector<int64_t> &hseg, int64_t *dseg) {
    const int nseg = static_cast<int>(hseg.size() / 2);
    if (nseg == 0) return KTG_OK;
    std::vector<int64_t> small;
    small.reserve(hseg.size());
    for (int s = 0; s < nseg; ++s) {
        const int64_t b = hseg[2 * s], e = hseg[2 * s + 1];
        if (e - b <= 1) continue;
        if (e - b <= kSortSmall) {
            small.push_back(b);
            small.push_back(e);
            continue;
        }
        k_sort_chunks<<<blocks_for(e - b, kSortSmall), kT, 0, c->stream>>>(keys, b, e);
        ++c->launches;
        Key *src = keys;
        Key *dst = tmp;
        for (int64_t run = kSortSmall; run < e - b; run *= 2) {
            k_merge_pass<<<blocks_for(e - b), kT, 0, c->stream>>>(src, dst, b, e, run);
            ++c->launches;
            std::swap(src, dst);
        }
        if (src != keys) {
            k_copy_keys<<<blocks_for(e - b), kT, 0, c->stream>>>(src, keys, b, e);
            ++c->launches;
        }
    }
    if (!small.empty()) {
        KTG_CUDA(c, cudaMemcpyAsync(dseg, small.data(), sizeof(int64_t) * small.size(),
                                    cudaMemcpyHostToDevice, c->stream));
        k_sort_small<<<static_cast<int>(small.size() / 2), kT, 0, c->stream>>>(
            keys, dseg, static_cast<int>(small.size() / 2));
        ++c->launches;
    }
    KTG_CUDA(c, cudaGetLastError());
    return KTG_OK;
}

// ---- free space -----------------------------------------------------------------

struct Free {
    const double *rowy;      // [2R] y start, y end (rows sorted by y start)
    const int64_t *rowspan;  // [R+1]
    const double *spans;     // [2S] x start, x end
    const double *obst;      // [4K] lx ly ux uy
    int32_t R, K;
};

// First row with ly < y.end (std::upper_bound with v < r.y.end).
__device__ __forceinline__ int32_t first_row(const Free &F, double ly) {
    int32_t lo = 0, hi = F.R;
    while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (ly < F.rowy[2 * mid + 1]) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// Upper bound on a profile's step count and edge count for `box`.
__device__ __forceinline__ void profile_bound(const Free &F, const double *box, bool vertical,
                                              int64_t &steps, int64_t &edges) {
    const int32_t r0 = first_row(F, box[1]);
    int32_t r1 = r0;
    while (r1 < F.R && F.rowy[2 * r1] < box[3]) ++r1;
    const int64_t sp = F.rowspan[r1] - F.rowspan[r0];
    steps = vertical ? 2 * sp : 0;
    edges = (vertical ? 2 * sp : 2 * static_cast<int64_t>(r1 - r0)) + 2;
}

// Vertical profile steps of `box` (unsorted), returns the count.
__device__ int64_t profile_steps(const Free &F, const double *box, Key *out) {
    const double lx = box[0], ly = box[1], ux = box[2], uy = box[3];
    int64_t k = 0;
    for (int32_t r = first_row(F, ly); r < F.R && F.rowy[2 * r] < uy; ++r) {
        const double h = ref_min(uy, F.rowy[2 * r + 1]) - ref_max(ly, F.rowy[2 * r]);
        for (int64_t s = F.rowspan[r]; s < F.rowspan[r + 1]; ++s) {
            const double a = ref_max(F.spans[2 * s], lx);
            const double z = ref_min(F.spans[2 * s + 1], ux);
            if (h > 0.0 && z > a) {
                out[k++] = Key{ord(a), ord(h)};
                out[k++] = Key{ord(z), ord(-h)};
            }
        }
    }
    return k;
}

// AxisProfile (simpl_grid.h:29-65, getProfile :179-232) stored as edges /
// prefix arrays of `n` entries.
struct Prof {
    const double *e;
    const double *p;
    int64_t n;
    __device__ double total() const { return p[n - 1]; }
    __device__ double before(double c) const {
        if (c <= e[0]) return 0.0;
        if (c >= e[n - 1]) return total();
        int64_t lo = 0, hi = n;  // upper_bound
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (c < e[mid]) hi = mid;
            else lo = mid + 1;
        }
        const int64_t k = lo - 1;
        const double f = (c - e[k]) / (e[k + 1] - e[k]);
        return p[k] + f * (p[k + 1] - p[k]);
    }
    __device__ double between(double a, double b) const { return before(b) - before(a); }
    __device__ double coordinate_at(double target) const {
        if (target <= 0.0) return e[0];
        if (target >= total()) return e[n - 1];
        int64_t lo = 0, hi = n;  // lower_bound on prefix
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (p[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        const int64_t k = lo;
        const double step = p[k] - p[k - 1];
        const double f = step > 0.0 ? (target - p[k - 1]) / step : 1.0;
        return e[k - 1] + f * (e[k] - e[k - 1]);
    }
};

// Builds the profile of `box` into e/p from its sorted steps (vertical) or
// the rows (horizontal); returns the number of edges.
__device__ int64_t build_profile(const Free &F, const double *box, bool vertical, const Key *steps,
                                 int64_t nsteps, double *e, double *p) {
    const double lx = box[0], ly = box[1], ux = box[2], uy = box[3];
    const double lo = vertical ? lx : ly, hi = vertical ? ux : uy;
    int64_t n = 1;
    e[0] = lo;
    p[0] = 0.0;
    auto extend = [&](double to, double area) {
        if (to > e[n - 1]) {
            e[n] = to;
            p[n] = p[n - 1] + area;
            ++n;
        }
    };
    if (vertical) {
        double height = 0.0;
        for (int64_t k = 0; k < nsteps; ++k) {
            const double at = unord(steps[k].a), dh = unord(steps[k].b);
            extend(at, height * (at - e[n - 1]));
            height += dh;
        }
    } else {
        for (int32_t r = first_row(F, ly); r < F.R && F.rowy[2 * r] < uy; ++r) {
            const double a = ref_max(lo, F.rowy[2 * r]);
            const double z = ref_min(hi, F.rowy[2 * r + 1]);
            if (z > a) {
                extend(a, 0.0);
                double total = 0.0;  // Row::getLength(b.getX())
                for (int64_t s = F.rowspan[r]; s < F.rowspan[r + 1]; ++s)
                    total += ref_max(0.0, ref_min(ux, F.spans[2 * s + 1]) - ref_max(lx, F.spans[2 * s]));
                extend(z, total * (z - a));
            }
        }
    }
    extend(hi, 0.0);
    if (n == 1) {
        e[1] = hi;
        p[1] = 0.0;
        n = 2;
    }
    return n;
}

// ---- per-level kernels --------------------------------------------------------------

struct CellsDev {
    double *x, *y;
    const double *w, *h, *area;
};

__device__ __forceinline__ double centre(const CellsDev &C, int32_t i, bool vertical) {
    return vertical ? C.x[i] + 0.5 * C.w[i] : C.y[i] + 0.5 * C.h[i];
}

struct Level {
    int32_t na;
    const int32_t *b, *e;  // cell ranges of the active blocks
    const double *box;     // [4 na]
    const int32_t *vert;
    const double *room;
    // results
    int32_t *m;
    double *low_area, *high_area, *cut;
    double *half_box;      // [8 na]: low box, high box
    int64_t *bound;        // [2 na] or [4 na]: steps, edges per owner
};

// The per-cell kernels below run on a 2-D grid: y strides over the active
// blocks, x over the cells of one block.
__global__ void k_centre_keys(Level L, CellsDev C, const int32_t *cells, Key *keys) {
    for (int32_t blk = blockIdx.y; blk < L.na; blk += gridDim.y) {
        const int32_t b = L.b[blk], e = L.e[blk];
        const bool v = L.vert[blk] != 0;
        for (int32_t p = b + blockIdx.x * blockDim.x + threadIdx.x; p < e; p += gridDim.x * blockDim.x) {
            const int32_t i = cells[p];
            keys[p] = Key{ord(centre(C, i, v)), static_cast<unsigned long long>(i)};
        }
    }
}

__global__ void k_keys_to_cells(Level L, const Key *keys, int32_t *cells) {
    for (int32_t blk = blockIdx.y; blk < L.na; blk += gridDim.y)
        for (int32_t p = L.b[blk] + blockIdx.x * blockDim.x + threadIdx.x; p < L.e[blk];
             p += gridDim.x * blockDim.x)
            cells[p] = static_cast<int32_t>(keys[p].b);
}

// One thread per block: areas and median in the reference's order, and the
// block profile's bound.
__global__ void k_block_split(Level L, CellsDev C, Free F, const int32_t *cells) {
    const int32_t blk = blockIdx.x * blockDim.x + threadIdx.x;
    if (blk >= L.na) return;
    const int32_t b = L.b[blk], e = L.e[blk];
    const int32_t size = e - b;
    double cell_area = 0.0;
    for (int32_t p = b; p < e; ++p) cell_area += C.area[cells[p]];
    int32_t m = 0;
    double low = 0.0;
    while (m + 1 < size && (m == 0 || low < 0.5 * cell_area)) low += C.area[cells[b + m++]];
    double high = 0.0;
    for (int32_t p = b + m; p < e; ++p) high += C.area[cells[p]];
    L.m[blk] = m;
    L.low_area[blk] = low;
    L.high_area[blk] = high;
    L.cut[blk] = cell_area;  // kept until the cutline replaces it
    int64_t st, ed;
    profile_bound(F, L.box + 4 * blk, L.vert[blk] != 0, st, ed);
    L.bound[2 * blk] = st;
    L.bound[2 * blk + 1] = ed;
}

__global__ void k_block_steps(Level L, Free F, const int64_t *soff, Key *steps, int64_t *nsteps) {
    const int32_t blk = blockIdx.x * blockDim.x + threadIdx.x;
    if (blk >= L.na) return;
    nsteps[blk] = L.vert[blk] ? profile_steps(F, L.box + 4 * blk, steps + soff[blk]) : 0;
}

// One thread per block: profile, cutline, half boxes, half bounds.
__global__ void k_block_cut(Level L, Free F, const int64_t *soff, const Key *steps,
                            const int64_t *nsteps, const int64_t *eoff, double *pe, double *pp,
                            int64_t *hbound) {
    const int32_t blk = blockIdx.x * blockDim.x + threadIdx.x;
    if (blk >= L.na) return;
    const bool v = L.vert[blk] != 0;
    const double *box = L.box + 4 * blk;
    double *e = pe + eoff[blk], *p = pp + eoff[blk];
    const int64_t n = build_profile(F, box, v, steps + soff[blk], nsteps[blk], e, p);
    const Prof room{e, p, n};
    const double cell_area = L.cut[blk];
    const double share = cell_area > 0.0 ? L.low_area[blk] / cell_area : 0.5;
    const double lo = v ? box[0] : box[1], hi = v ? box[2] : box[3];
    const double cut = room.total() > 0.0 ? room.coordinate_at(share * room.total())
                                          : lo + share * (hi - lo);
    L.cut[blk] = cut;
    double *lb = L.half_box + 8 * blk, *hb = lb + 4;
    for (int k = 0; k < 4; ++k) lb[k] = hb[k] = box[k];
    (v ? lb[2] : lb[3]) = cut;
    (v ? hb[0] : hb[1]) = cut;
    for (int side = 0; side < 2; ++side) {
        const double *bx = side ? hb : lb;
        int64_t st, ed;
        profile_bound(F, bx, v, st, ed);
        int64_t k = 0;  // obstacles overlapping the half box
        for (int32_t o = 0; o < F.K; ++o) {
            const double *ob = F.obst + 4 * o;
            if (ob[2] <= bx[0] || ob[0] >= bx[2] || ob[3] <= bx[1] || ob[1] >= bx[3]) continue;
            ++k;
        }
        hbound[4 * blk + 2 * side] = st;
        hbound[4 * blk + 2 * side + 1] = ed + 2 * k + 2 + 256;  // profile edges, then cuts
    }
}

__global__ void k_half_steps(Level L, Free F, const int64_t *soff, Key *steps, int64_t *nsteps) {
    const int32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 2 * L.na) return;
    const int32_t blk = h >> 1;
    nsteps[h] = L.vert[blk] ? profile_steps(F, L.half_box + 4 * h, steps + soff[h]) : 0;
}

struct Stripes {
    int64_t *off;    // [2 na] first stripe of the half (into the arrays below)
    int32_t *count;  // [2 na]
    double *a, *b, *cap, *used;
    unsigned long long *lo, *hi;
};

// One thread per half: profile, stripes (getStripes, simpl_lal.cc:265-308),
// ordered by distance from the cut (stable, farthest first).
__global__ void k_half_stripes(Level L, Free F, const int64_t *soff, const Key *steps,
                               const int64_t *nsteps, const int64_t *eoff, double *pe, double *pp,
                               int64_t *cap_over, double frac, double limit_density, Stripes S,
                               int *status) {
    const int32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 2 * L.na) return;
    const int32_t blk = h >> 1;
    const int side = h & 1;
    const bool v = L.vert[blk] != 0;
    const double *box = L.half_box + 4 * h;
    double *e = pe + eoff[h], *p = pp + eoff[h];
    const int64_t n = build_profile(F, box, v, steps + soff[h], nsteps[h], e, p);
    const Prof room{e, p, n};
    const double cell_area = side ? L.high_area[blk] : L.low_area[blk];
    const double region_room = L.room[blk];
    const double lo = v ? box[0] : box[1], hi = v ? box[2] : box[3];
    // cuts live after the profile in the same scratch
    double *cuts = p + n;
    const int64_t cap = cap_over[h];  // cuts (and stripes) the half may hold
    int64_t nc = 0;
    cuts[nc++] = lo;
    cuts[nc++] = hi;
    for (int32_t o = 0; o < F.K; ++o) {
        const double *ob = F.obst + 4 * o;
        if (ob[2] <= box[0] || ob[0] >= box[2] || ob[3] <= box[1] || ob[1] >= box[3]) continue;
        const double e0 = v ? ob[0] : ob[1], e1 = v ? ob[2] : ob[3];
        if (e0 > lo && e0 < hi) cuts[nc++] = e0;
        if (e1 > lo && e1 < hi) cuts[nc++] = e1;
    }
    for (int64_t i = 1; i < nc; ++i) {  // insertion sort (stable)
        const double t = cuts[i];
        int64_t j = i - 1;
        while (j >= 0 && t < cuts[j]) {
            cuts[j + 1] = cuts[j];
            --j;
        }
        cuts[j + 1] = t;
    }
    int64_t u = 0;
    for (int64_t i = 0; i < nc; ++i)
        if (u == 0 || !(cuts[u - 1] == cuts[i])) cuts[u++] = cuts[i];
    nc = u;
    const double limit = frac * (region_room > 0.0 ? region_room : room.total());
    const double fill = room.total() > 0.0 ? ref_min(limit_density, cell_area / room.total())
                                           : limit_density;
    for (int64_t s = 0; s + 1 < nc;) {
        const double a = cuts[s], b = cuts[s + 1];
        const double here = room.between(a, b);
        const double mid = room.coordinate_at(room.before(a) + 0.5 * here);
        if (here > limit && mid > a && mid < b) {
            if (nc + 1 > cap) {
                atomicCAS(status, kStatusOk, kStatusCapacity);
                break;
            }
            for (int64_t q = nc; q > s + 1; --q) cuts[q] = cuts[q - 1];
            cuts[s + 1] = mid;
            ++nc;
        } else {
            ++s;
        }
    }
    const int64_t ns = nc - 1;
    const int64_t so = S.off[h];
    const double cutline = L.cut[blk];
    const bool below = side == 0;
    for (int64_t s = 0; s < ns; ++s) {
        S.a[so + s] = cuts[s];
        S.b[so + s] = cuts[s + 1];
        S.cap[so + s] = fill * room.between(cuts[s], cuts[s + 1]);
    }
    // stable sort by fromCut(center) descending (insertion sort on the arrays)
    for (int64_t i = 1; i < ns; ++i) {
        const double ta = S.a[so + i], tb = S.b[so + i], tc = S.cap[so + i];
        const double cc = 0.5 * (ta + tb);
        const double fc = below ? cutline - cc : cc - cutline;
        int64_t j = i - 1;
        while (j >= 0) {
            const double cj = 0.5 * (S.a[so + j] + S.b[so + j]);
            const double fj = below ? cutline - cj : cj - cutline;
            if (!(fc > fj)) break;
            S.a[so + j + 1] = S.a[so + j];
            S.b[so + j + 1] = S.b[so + j];
            S.cap[so + j + 1] = S.cap[so + j];
            --j;
        }
        S.a[so + j + 1] = ta;
        S.b[so + j + 1] = tb;
        S.cap[so + j + 1] = tc;
    }
    for (int64_t s = 0; s < ns; ++s) {
        S.used[so + s] = 0.0;
        S.lo[so + s] = ~0ull;
        S.hi[so + s] = 0ull;
    }
    S.count[h] = static_cast<int32_t>(ns);
}

__global__ void k_fill_keys(Level L, CellsDev C, const int32_t *cells, Key *keys) {
    for (int32_t blk = blockIdx.y; blk < L.na; blk += gridDim.y) {
        const int32_t b = L.b[blk], e = L.e[blk], mid = b + L.m[blk];
        const bool v = L.vert[blk] != 0;
        const double cut = L.cut[blk];
        for (int32_t p = b + blockIdx.x * blockDim.x + threadIdx.x; p < e; p += gridDim.x * blockDim.x) {
            const int32_t i = cells[p];
            const double c = centre(C, i, v);
            const double from = p < mid ? cut - c : c - cut;
            keys[p] = Key{ord(-from), static_cast<unsigned long long>(i)};
        }
    }
}

// One thread per half: greedy fill in the sorted order (nonlinearScale,
// simpl_lal.cc:332-340).
__global__ void k_fill(Level L, CellsDev C, const int32_t *cells, Stripes S, int32_t *stripe_of) {
    const int32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 2 * L.na) return;
    const int32_t blk = h >> 1;
    const int32_t b = L.b[blk], e = L.e[blk], mid = b + L.m[blk];
    const int32_t p0 = (h & 1) ? mid : b, p1 = (h & 1) ? e : mid;
    const int64_t so = S.off[h];
    const int32_t ns = S.count[h];
    if (ns == 0) {  // a half of zero width: its cells stay where they are
        for (int32_t p = p0; p < p1; ++p) stripe_of[cells[p]] = -1;
        return;
    }
    int32_t s = 0;
    for (int32_t p = p0; p < p1; ++p) {
        while (s + 1 < ns && S.used[so + s] >= S.cap[so + s]) ++s;
        const int32_t i = cells[p];
        stripe_of[i] = static_cast<int32_t>(so + s);
        S.used[so + s] += C.area[i];
    }
}

__global__ void k_stripe_minmax(Level L, CellsDev C, const int32_t *cells, Stripes S,
                                const int32_t *stripe_of) {
    for (int32_t blk = blockIdx.y; blk < L.na; blk += gridDim.y) {
        const int32_t b = L.b[blk], e = L.e[blk];
        const bool v = L.vert[blk] != 0;
        for (int32_t p = b + blockIdx.x * blockDim.x + threadIdx.x; p < e; p += gridDim.x * blockDim.x) {
            const int32_t i = cells[p];
            const int32_t s = stripe_of[i];
            if (s < 0) continue;
            const unsigned long long o = ord(centre(C, i, v));
            atomicMin(S.lo + s, o);
            atomicMax(S.hi + s, o);
        }
    }
}

__global__ void k_new_pos(Level L, CellsDev C, const int32_t *cells, Stripes S,
                          const int32_t *stripe_of) {
    for (int32_t blk = blockIdx.y; blk < L.na; blk += gridDim.y) {
    const int32_t b = L.b[blk], e = L.e[blk];
    const bool v = L.vert[blk] != 0;
    for (int32_t p = b + blockIdx.x * blockDim.x + threadIdx.x; p < e; p += gridDim.x * blockDim.x) {
        const int32_t i = cells[p];
        const int32_t s = stripe_of[i];
        if (s < 0) continue;
        const double lo = unord(S.lo[s]), hi = unord(S.hi[s]);
        const double c0 = centre(C, i, v);
        const double t = hi > lo ? (c0 - lo) / (hi - lo) : 0.5;
        const double size = v ? C.w[i] : C.h[i];
        const double a = S.a[s], bb = S.b[s];
        const double c = a + t * (bb - a);
        const double lim = ref_max(a, bb - size);
        double np = c - 0.5 * size;
        np = np < a ? a : (lim < np ? lim : np);  // std::clamp
        (v ? C.x : C.y)[i] = np;
    }
    }
}

// ---- batch set-up and bins ---------------------------------------------------------

struct GridDev {
    double ox, oy, dx, dy;
    int32_t nx, ny;
};

__device__ __forceinline__ int32_t clamp_index(double f, int32_t n) {
    const double hi = static_cast<double>(n) - 1e-9;
    const double c = f < 0.0 ? 0.0 : (hi < f ? hi : f);
    return static_cast<int32_t>(c);
}

__global__ void k_bins(CellsDev C, int32_t n, GridDev G, int32_t *binof) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t ix = clamp_index((C.x[i] + 0.5 * C.w[i] - G.ox) / G.dx, G.nx);
    const int32_t iy = clamp_index((C.y[i] + 0.5 * C.h[i] - G.oy) / G.dy, G.ny);
    binof[i] = iy * G.nx + ix;
}

__global__ void k_region_map(const int32_t *rects, int32_t nreg, int32_t nx, int32_t *map) {
    for (int32_t r = blockIdx.y; r < nreg; r += gridDim.y) {
        const int32_t x0 = rects[4 * r], x1 = rects[4 * r + 1], y0 = rects[4 * r + 2],
                      y1 = rects[4 * r + 3];
        const int64_t w = x1 - x0 + 1, cnt = w * (y1 - y0 + 1);
        for (int64_t k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x)
            map[(y0 + k / w) * nx + x0 + k % w] = r;
    }
}

__global__ void k_region_count(const int32_t *binof, int32_t n, const int32_t *map, int32_t *cnt) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t r = map[binof[i]];
    if (r >= 0) atomicAdd(cnt + r, 1);
}

__global__ void k_region_place(const int32_t *binof, int32_t n, const int32_t *map, int32_t *cursor,
                               int32_t *cells) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t r = map[binof[i]];
    if (r >= 0) cells[atomicAdd(cursor + r, 1)] = i;
}

__global__ void k_clamp_die(CellsDev C, int32_t n, double lx, double ly, double ux, double uy) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double mx = ref_max(lx, ux - C.w[i]), my = ref_max(ly, uy - C.h[i]);
    double x = C.x[i], y = C.y[i];
    x = x < lx ? lx : (mx < x ? mx : x);
    y = y < ly ? ly : (my < y ? my : y);
    C.x[i] = x;
    C.y[i] = y;
}

template <typename T>
struct DevBuf {
    T *p = nullptr;
    int64_t cap = 0;
    int ensure(ktg_ctx *c, int64_t n) {
        if (n <= cap) return KTG_OK;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const int64_t want = std::max<int64_t>(n + n / 4, 64);
        if (cudaMalloc(&p, sizeof(T) * want) != cudaSuccess)
            return set_error(c, KTG_ERR_NOMEM, "out of device memory (legalization)");
        cap = want;
        return KTG_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

}  // namespace

// Free space, obstacles and die for the legalizer, and its scratch.
struct LalState {
    std::vector<double> rowy, spans, obst;
    std::vector<int64_t> rowspan;
    double die[4] = {0, 0, 0, 0};
    DevBuf<double> d_rowy, d_spans, d_obst;
    DevBuf<int64_t> d_rowspan;
    DevBuf<int32_t> binof, map, cells, cnt, stripe_of, rects, lb, le, lvert, nb_, ne_, nvert;
    DevBuf<double> occ, lbox, lroom, nbox, nroom, low_area, high_area, cut, half_box;
    DevBuf<int32_t> m;
    DevBuf<int64_t> bound, hbound, soff, eoff, nsteps, hsoff, heoff, hnsteps, seg, stoff;
    DevBuf<Key> keys, keys_tmp, steps, steps_tmp;
    DevBuf<double> pe, pp;
    DevBuf<int32_t> scount;
    DevBuf<double> sa, sb, scap, sused;
    DevBuf<unsigned long long> slo, shi;
    DevBuf<double> overflow;
};

void free_lal(ktg_ctx *c) {
    LalState *s = c->lal;
    if (!s) return;
    for (auto *b : {&s->binof, &s->map, &s->cells, &s->cnt, &s->stripe_of, &s->rects, &s->lb,
                    &s->le, &s->lvert, &s->nb_, &s->ne_, &s->nvert, &s->m, &s->scount})
        b->release();
    for (auto *b : {&s->d_rowy, &s->d_spans, &s->d_obst, &s->occ, &s->lbox, &s->lroom, &s->nbox,
                    &s->nroom, &s->low_area, &s->high_area, &s->cut, &s->half_box, &s->pe, &s->pp,
                    &s->sa, &s->sb, &s->scap, &s->sused, &s->overflow})
        b->release();
    for (auto *b : {&s->d_rowspan, &s->bound, &s->hbound, &s->soff, &s->eoff, &s->nsteps,
                    &s->hsoff, &s->heoff, &s->hnsteps, &s->seg, &s->stoff})
        b->release();
    s->keys.release();
    s->keys_tmp.release();
    s->steps.release();
    s->steps_tmp.release();
    s->slo.release();
    s->shi.release();
    delete s;
    c->lal = nullptr;
}

int set_free_space(ktg_ctx *c, int64_t nrows, const double *rowy, const int64_t *rowspan,
                   const double *spans, int64_t nobst, const double *obst, const double *die4) {
    if (!c->lal) c->lal = new LalState();
    LalState *s = c->lal;
    const int64_t S = nrows > 0 ? rowspan[nrows] : 0;
    s->rowy.assign(rowy, rowy + 2 * nrows);
    s->rowspan.assign(rowspan, rowspan + nrows + 1);
    s->spans.assign(spans, spans + 2 * S);
    s->obst.assign(obst, obst + 4 * nobst);
    std::copy(die4, die4 + 4, s->die);
    int rc;
    if ((rc = s->d_rowy.ensure(c, 2 * nrows + 2)) || (rc = s->d_rowspan.ensure(c, nrows + 2)) ||
        (rc = s->d_spans.ensure(c, 2 * S + 2)) || (rc = s->d_obst.ensure(c, 4 * nobst + 4)))
        return rc;
    KTG_CUDA(c, cudaMemcpyAsync(s->d_rowy.p, s->rowy.data(), sizeof(double) * s->rowy.size(),
                                cudaMemcpyHostToDevice, c->stream));
    KTG_CUDA(c, cudaMemcpyAsync(s->d_rowspan.p, s->rowspan.data(),
                                sizeof(int64_t) * s->rowspan.size(), cudaMemcpyHostToDevice, c->stream));
    if (S > 0)
        KTG_CUDA(c, cudaMemcpyAsync(s->d_spans.p, s->spans.data(), sizeof(double) * s->spans.size(),
                                    cudaMemcpyHostToDevice, c->stream));
    if (nobst > 0)
        KTG_CUDA(c, cudaMemcpyAsync(s->d_obst.p, s->obst.data(), sizeof(double) * s->obst.size(),
                                    cudaMemcpyHostToDevice, c->stream));
    KTG_CUDA(c, cudaStreamSynchronize(c->stream));
    return KTG_OK;
}

namespace {

// ---- host side: clusters and growth exactly as the reference sums them ---------------

struct HostGrid {
    int32_t nx, ny;
    const std::vector<double> *avail;
    double limit;
    double rect_sum(const std::vector<double> &f, const int32_t *r) const {
        double t = 0.0;
        for (int32_t iy = r[2]; iy <= r[3]; ++iy)
            for (int32_t ix = r[0]; ix <= r[1]; ++ix) t += f[static_cast<size_t>(iy) * nx + ix];
        return t;
    }
    double density(const std::vector<double> &occ, const int32_t *r) const {
        const double cells = rect_sum(occ, r);
        const double room = rect_sum(*avail, r);
        if (room > 0.0) return cells / room;
        return cells > 0.0 ? std::numeric_limits<double>::infinity() : 0.0;
    }
    std::vector<std::array<int32_t, 4>> clusters(const std::vector<double> &occ) const {
        const int64_t N = static_cast<int64_t>(nx) * ny;
        std::vector<char> over(N);
        for (int64_t k = 0; k < N; ++k) over[k] = occ[k] > limit * (*avail)[k] ? 1 : 0;
        std::vector<std::array<int32_t, 4>> out;
        std::vector<int64_t> frontier;
        for (int64_t seed = 0; seed < N; ++seed) {
            if (!over[seed]) continue;
            over[seed] = 0;
            frontier.assign(1, seed);
            std::array<int32_t, 4> r{static_cast<int32_t>(seed % nx), static_cast<int32_t>(seed % nx),
                                     static_cast<int32_t>(seed / nx), static_cast<int32_t>(seed / nx)};
            while (!frontier.empty()) {
                const int64_t k = frontier.back();
                frontier.pop_back();
                const int32_t ix = static_cast<int32_t>(k % nx), iy = static_cast<int32_t>(k / nx);
                r[0] = std::min(r[0], ix);
                r[1] = std::max(r[1], ix);
                r[2] = std::min(r[2], iy);
                r[3] = std::max(r[3], iy);
                const int32_t st[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};
                for (const auto &d : st) {
                    const int64_t px = ix + d[0], py = iy + d[1];
                    if (px < 0 || py < 0 || px >= nx || py >= ny) continue;
                    const int64_t kk = py * nx + px;
                    if (over[kk]) {
                        over[kk] = 0;
                        frontier.push_back(kk);
                    }
                }
            }
            out.push_back(r);
        }
        return out;
    }
    std::array<int32_t, 4> grown(std::array<int32_t, 4> r, const std::vector<double> &occ) const {
        while (density(occ, r.data()) > limit) {
            const std::array<std::array<int32_t, 4>, 4> wider{{
                {r[0] > 0 ? r[0] - 1 : r[0], r[1], r[2], r[3]},
                {r[0], r[1] + 1 < nx ? r[1] + 1 : r[1], r[2], r[3]},
                {r[0], r[1], r[2] > 0 ? r[2] - 1 : r[2], r[3]},
                {r[0], r[1], r[2], r[3] + 1 < ny ? r[3] + 1 : r[3]},
            }};
            const int64_t bins = static_cast<int64_t>(r[1] - r[0] + 1) * (r[3] - r[2] + 1);
            int best = -1;
            double best_d = std::numeric_limits<double>::infinity();
            for (int k = 0; k < 4; ++k) {
                const auto &w = wider[k];
                if (static_cast<int64_t>(w[1] - w[0] + 1) * (w[3] - w[2] + 1) == bins) continue;
                const double d = density(occ, w.data());
                if (best < 0 || d < best_d) {
                    best = k;
                    best_d = d;
                }
            }
            if (best < 0) break;
            r = wider[best];
        }
        return r;
    }
};

}  // namespace

// Runs the legalizer on positions x, y (device, n values) in place.
int launch_lal(ktg_ctx *c, double *x, double *y, int32_t max_level, int32_t min_cells,
               double frac) {
    LalState *s = c->lal;
    const int32_t n = static_cast<int32_t>(c->n);
    const int32_t nx = static_cast<int32_t>(c->nx), ny = static_cast<int32_t>(c->ny);
    const int64_t nbins = static_cast<int64_t>(nx) * ny;
    int rc;
    if ((rc = s->binof.ensure(c, n + 1)) || (rc = s->map.ensure(c, nbins)) ||
        (rc = s->cells.ensure(c, n + 1)) || (rc = s->stripe_of.ensure(c, n + 1)) ||
        (rc = s->occ.ensure(c, nbins)) || (rc = s->overflow.ensure(c, 1)) ||
        (rc = s->keys.ensure(c, n + 1)) || (rc = s->keys_tmp.ensure(c, n + 1)))
        return rc;
    KTG_CUDA(c, cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
    CellsDev C{x, y, c->width, c->height, c->area};
    const GridDev G{c->origin_x, c->origin_y, c->dx, c->dy, nx, ny};
    Free F{s->d_rowy.p, s->d_rowspan.p, s->d_spans.p, s->d_obst.p,
           static_cast<int32_t>(s->rowy.size() / 2), static_cast<int32_t>(s->obst.size() / 4)};
    const HostGrid HG{nx, ny, &c->avail_host, c->density_limit};
    std::vector<double> occ(nbins);
    auto refresh = [&]() -> int {  // bins and occupancy of the current positions
        if (n > 0) {
            k_bins<<<blocks_for(n), kT, 0, c->stream>>>(C, n, G, s->binof.p);
            ++c->launches;
        }
        int r2 = launch_occupancy(c, x, y, s->occ.p, s->overflow.p);
        if (r2) return r2;
        KTG_CUDA(c, cudaMemcpyAsync(occ.data(), s->occ.p, sizeof(double) * nbins,
                                    cudaMemcpyDeviceToHost, c->stream));
        KTG_CUDA(c, cudaStreamSynchronize(c->stream));
        return KTG_OK;
    };
    if ((rc = refresh())) return rc;

    auto reach = [&](const std::array<int32_t, 4> &r) {
        return std::array<int32_t, 4>{r[0] > 0 ? r[0] - 1 : 0, std::min(r[1] + 1, nx - 1),
                                      r[2] > 0 ? r[2] - 1 : 0, std::min(r[3] + 1, ny - 1)};
    };
    auto touches = [](const std::array<int32_t, 4> &a, const std::array<int32_t, 4> &b) {
        return a[0] <= b[1] && b[0] <= a[1] && a[2] <= b[3] && b[2] <= a[3];
    };
    std::vector<std::array<int32_t, 4>> batch, batch_reach;

    auto run_batch = [&]() -> int {
        const int32_t nreg = static_cast<int32_t>(batch.size());
        if (nreg == 0) return KTG_OK;
        int r2;
        std::vector<int32_t> rects(4 * nreg);
        std::vector<double> box(4 * nreg), room(nreg);
        for (int32_t r = 0; r < nreg; ++r) {
            for (int k = 0; k < 4; ++k) rects[4 * r + k] = batch[r][k];
            box[4 * r + 0] = c->origin_x + static_cast<double>(batch[r][0]) * c->dx;
            box[4 * r + 1] = c->origin_y + static_cast<double>(batch[r][2]) * c->dy;
            box[4 * r + 2] = c->origin_x + static_cast<double>(batch[r][1] + 1) * c->dx;
            box[4 * r + 3] = c->origin_y + static_cast<double>(batch[r][3] + 1) * c->dy;
            room[r] = HG.rect_sum(c->avail_host, batch[r].data());
        }
        if ((r2 = s->rects.ensure(c, 4 * nreg)) || (r2 = s->cnt.ensure(c, nreg + 1))) return r2;
        KTG_CUDA(c, cudaMemcpyAsync(s->rects.p, rects.data(), sizeof(int32_t) * rects.size(),
                                    cudaMemcpyHostToDevice, c->stream));
        KTG_CUDA(c, cudaMemsetAsync(s->map.p, 0xff, sizeof(int32_t) * nbins, c->stream));
        KTG_CUDA(c, cudaMemsetAsync(s->cnt.p, 0, sizeof(int32_t) * (nreg + 1), c->stream));
        k_region_map<<<dim3(64, std::min(nreg, 65535)), kT, 0, c->stream>>>(s->rects.p, nreg, nx, s->map.p);
        k_region_count<<<blocks_for(n), kT, 0, c->stream>>>(s->binof.p, n, s->map.p, s->cnt.p);
        c->launches += 2;
        std::vector<int32_t> cnt(nreg);
        KTG_CUDA(c, cudaMemcpyAsync(cnt.data(), s->cnt.p, sizeof(int32_t) * nreg,
                                    cudaMemcpyDeviceToHost, c->stream));
        KTG_CUDA(c, cudaStreamSynchronize(c->stream));
        // level-1 blocks: one per region
        std::vector<int32_t> hb(nreg), he(nreg), hv(nreg, 1);
        int32_t run = 0;
        for (int32_t r = 0; r < nreg; ++r) {
            hb[r] = run;
            run += cnt[r];
            he[r] = run;
        }
        if ((r2 = s->lb.ensure(c, nreg)) || (r2 = s->le.ensure(c, nreg)) ||
            (r2 = s->lvert.ensure(c, nreg)) || (r2 = s->lbox.ensure(c, 4 * nreg)) ||
            (r2 = s->lroom.ensure(c, nreg)))
            return r2;
        KTG_CUDA(c, cudaMemcpyAsync(s->cnt.p, hb.data(), sizeof(int32_t) * nreg,
                                    cudaMemcpyHostToDevice, c->stream));
        k_region_place<<<blocks_for(n), kT, 0, c->stream>>>(s->binof.p, n, s->map.p, s->cnt.p,
                                                             s->cells.p);
        ++c->launches;
        // host copies of the current level's blocks
        std::vector<double> hbox = box, hroom = room;
        for (int32_t level = 1; level < max_level; ++level) {
            // active blocks: more than min_cells cells
            std::vector<int32_t> ab, ae, av;
            std::vector<double> abox, aroom;
            for (size_t k = 0; k < hb.size(); ++k) {
                if (he[k] - hb[k] <= min_cells) continue;
                ab.push_back(hb[k]);
                ae.push_back(he[k]);
                av.push_back(hv[k]);
                for (int q = 0; q < 4; ++q) abox.push_back(hbox[4 * k + q]);
                aroom.push_back(hroom[k]);
            }
            const int32_t na = static_cast<int32_t>(ab.size());
            if (na == 0) break;
            if ((r2 = s->lb.ensure(c, na)) || (r2 = s->le.ensure(c, na)) ||
                (r2 = s->lvert.ensure(c, na)) || (r2 = s->lbox.ensure(c, 4 * na)) ||
                (r2 = s->lroom.ensure(c, na)) || (r2 = s->m.ensure(c, na)) ||
                (r2 = s->low_area.ensure(c, na)) || (r2 = s->high_area.ensure(c, na)) ||
                (r2 = s->cut.ensure(c, na)) || (r2 = s->half_box.ensure(c, 8 * na)) ||
                (r2 = s->bound.ensure(c, 2 * na)) || (r2 = s->hbound.ensure(c, 4 * na)) ||
                (r2 = s->soff.ensure(c, na)) || (r2 = s->eoff.ensure(c, na)) ||
                (r2 = s->nsteps.ensure(c, na)) || (r2 = s->hsoff.ensure(c, 2 * na)) ||
                (r2 = s->heoff.ensure(c, 2 * na)) || (r2 = s->hnsteps.ensure(c, 2 * na)) ||
                (r2 = s->seg.ensure(c, 4 * na + 2)) || (r2 = s->stoff.ensure(c, 2 * na)) ||
                (r2 = s->scount.ensure(c, 2 * na)))
                return r2;
            KTG_CUDA(c, cudaMemcpyAsync(s->lb.p, ab.data(), sizeof(int32_t) * na, cudaMemcpyHostToDevice, c->stream));
            KTG_CUDA(c, cudaMemcpyAsync(s->le.p, ae.data(), sizeof(int32_t) * na, cudaMemcpyHostToDevice, c->stream));
            KTG_CUDA(c, cudaMemcpyAsync(s->lvert.p, av.data(), sizeof(int32_t) * na, cudaMemcpyHostToDevice, c->stream));
            KTG_CUDA(c, cudaMemcpyAsync(s->lbox.p, abox.data(), sizeof(double) * 4 * na, cudaMemcpyHostToDevice, c->stream));
            KTG_CUDA(c, cudaMemcpyAsync(s->lroom.p, aroom.data(), sizeof(double) * na, cudaMemcpyHostToDevice, c->stream));
            Level L{na, s->lb.p, s->le.p, s->lbox.p, s->lvert.p, s->lroom.p, s->m.p, s->low_area.p,
                    s->high_area.p, s->cut.p, s->half_box.p, s->bound.p};
            int32_t maxlen = 0;
            std::vector<int64_t> segs(2 * na);
            for (int32_t k = 0; k < na; ++k) {
                maxlen = std::max(maxlen, ae[k] - ab[k]);
                segs[2 * k] = ab[k];
                segs[2 * k + 1] = ae[k];
            }
            const dim3 gcell(std::min(64, blocks_for(maxlen)), std::min(na, 65535));
            // 1. cells by centre
            k_centre_keys<<<gcell, kT, 0, c->stream>>>(L, C, s->cells.p, s->keys.p);
            ++c->launches;
            if ((r2 = seg_sort(c, s->keys.p, s->keys_tmp.p, segs, s->seg.p))) return r2;
            k_keys_to_cells<<<gcell, kT, 0, c->stream>>>(L, s->keys.p, s->cells.p);
            // 2. areas, median, block profile bounds
            k_block_split<<<blocks_for(na), kT, 0, c->stream>>>(L, C, F, s->cells.p);
            c->launches += 2;
            std::vector<int64_t> bound(2 * na);
            KTG_CUDA(c, cudaMemcpyAsync(bound.data(), s->bound.p, sizeof(int64_t) * 2 * na,
                                        cudaMemcpyDeviceToHost, c->stream));
            KTG_CUDA(c, cudaStreamSynchronize(c->stream));
            std::vector<int64_t> soff(na), eoff(na);
            int64_t st = 0, ed = 0;
            for (int32_t k = 0; k < na; ++k) {
                soff[k] = st;
                st += bound[2 * k];
                eoff[k] = ed;
                ed += bound[2 * k + 1];
            }
            if ((r2 = s->steps.ensure(c, st + 1)) || (r2 = s->steps_tmp.ensure(c, st + 1)) ||
                (r2 = s->pe.ensure(c, ed + 1)) || (r2 = s->pp.ensure(c, ed + 1)))
                return r2;
            KTG_CUDA(c, cudaMemcpyAsync(s->soff.p, soff.data(), sizeof(int64_t) * na, cudaMemcpyHostToDevice, c->stream));
            KTG_CUDA(c, cudaMemcpyAsync(s->eoff.p, eoff.data(), sizeof(int64_t) * na, cudaMemcpyHostToDevice, c->stream));
            k_block_steps<<<blocks_for(na), kT, 0, c->stream>>>(L, F, s->soff.p, s->steps.p, s->nsteps.p);
            ++c->launches;
            std::vector<int64_t> nst(na);
            KTG_CUDA(c, cudaMemcpyAsync(nst.data(), s->nsteps.p, sizeof(int64_t) * na,
                                        cudaMemcpyDeviceToHost, c->stream));
            KTG_CUDA(c, cudaStreamSynchronize(c->stream));
            std::vector<int64_t> ssegs;
            for (int32_t k = 0; k < na; ++k) {
                ssegs.push_back(soff[k]);
                ssegs.push_back(soff[k] + nst[k]);
            }
            if ((r2 = seg_sort(c, s->steps.p, s->steps_tmp.p, ssegs, s->seg.p))) return r2;
            // 3. profile, cutline, half boxes and bounds
            k_block_cut<<<blocks_for(na), kT, 0, c->stream>>>(L, F, s->soff.p, s->steps.p, s->nsteps.p,
                                                            s->eoff.p, s->pe.p, s->pp.p, s->hbound.p);
            ++c->launches;
            std::vector<int64_t> hbound(4 * na);
            KTG_CUDA(c, cudaMemcpyAsync(hbound.data(), s->hbound.p, sizeof(int64_t) * 4 * na,
                                        cudaMemcpyDeviceToHost, c->stream));
            KTG_CUDA(c, cudaStreamSynchronize(c->stream));
            std::vector<int64_t> hsoff(2 * na), heoff(2 * na), hcap(2 * na), stoff(2 * na);
            st = ed = 0;
            int64_t stripes = 0;
            for (int32_t h = 0; h < 2 * na; ++h) {
                hsoff[h] = st;
                st += hbound[2 * h];
                heoff[h] = ed;
                // pe: the profile edges; pp: the prefix, then up to `edges` cuts
                const int64_t edges = hbound[2 * h + 1];
                hcap[h] = edges;
                ed += 2 * edges;
                stoff[h] = stripes;
                stripes += edges;
            }
            if ((r2 = s->steps.ensure(c, st + 1)) || (r2 = s->steps_tmp.ensure(c, st + 1)) ||
                (r2 = s->pe.ensure(c, ed + 1)) || (r2 = s->pp.ensure(c, ed + 1)) ||
                (r2 = s->sa.ensure(c, stripes + 1)) || (r2 = s->sb.ensure(c, stripes + 1)) ||
                (r2 = s->scap.ensure(c, stripes + 1)) || (r2 = s->sused.ensure(c, stripes + 1)) ||
                (r2 = s->slo.ensure(c, stripes + 1)) || (r2 = s->shi.ensure(c, stripes + 1)) ||
                (r2 = s->bound.ensure(c, 2 * na)))
                return r2;
            KTG_CUDA(c, cudaMemcpyAsync(s->hsoff.p, hsoff.data(), sizeof(int64_t) * 2 * na, cudaMemcpyHostToDevice, c->stream));
            KTG_CUDA(c, cudaMemcpyAsync(s->heoff.p, heoff.data(), sizeof(int64_t) * 2 * na, cudaMemcpyHostToDevice, c->stream));
            KTG_CUDA(c, cudaMemcpyAsync(s->stoff.p, stoff.data(), sizeof(int64_t) * 2 * na, cudaMemcpyHostToDevice, c->stream));
            // cut capacity per half, read by k_half_stripes
            KTG_CUDA(c, cudaMemcpyAsync(s->hbound.p, hcap.data(), sizeof(int64_t) * 2 * na, cudaMemcpyHostToDevice, c->stream));
            k_half_steps<<<blocks_for(2 * na), kT, 0, c->stream>>>(L, F, s->hsoff.p, s->steps.p, s->hnsteps.p);
            ++c->launches;
            std::vector<int64_t> hnst(2 * na);
            KTG_CUDA(c, cudaMemcpyAsync(hnst.data(), s->hnsteps.p, sizeof(int64_t) * 2 * na,
                                        cudaMemcpyDeviceToHost, c->stream));
            KTG_CUDA(c, cudaStreamSynchronize(c->stream));
            ssegs.clear();
            for (int32_t h = 0; h < 2 * na; ++h) {
                ssegs.push_back(hsoff[h]);
                ssegs.push_back(hsoff[h] + hnst[h]);
            }
            if ((r2 = seg_sort(c, s->steps.p, s->steps_tmp.p, ssegs, s->seg.p))) return r2;
            // 4. stripes per half (profile arrays: e in pe, p and the cuts in pp)
            Stripes S{s->stoff.p, s->scount.p, s->sa.p, s->sb.p, s->scap.p, s->sused.p, s->slo.p, s->shi.p};
            k_half_stripes<<<blocks_for(2 * na), kT, 0, c->stream>>>(
                L, F, s->hsoff.p, s->steps.p, s->hnsteps.p, s->heoff.p, s->pe.p, s->pp.p,
                s->hbound.p, frac, c->density_limit, S, c->status);
            // 5. fill order, fill, stripe ranges, positions
            k_fill_keys<<<gcell, kT, 0, c->stream>>>(L, C, s->cells.p, s->keys.p);
            c->launches += 2;
            std::vector<int32_t> mh(na);
            KTG_CUDA(c, cudaMemcpyAsync(mh.data(), s->m.p, sizeof(int32_t) * na,
                                        cudaMemcpyDeviceToHost, c->stream));
            std::vector<double> cuth(na);
            KTG_CUDA(c, cudaMemcpyAsync(cuth.data(), s->cut.p, sizeof(double) * na,
                                        cudaMemcpyDeviceToHost, c->stream));
            KTG_CUDA(c, cudaStreamSynchronize(c->stream));
            std::vector<int64_t> fsegs;
            for (int32_t k = 0; k < na; ++k) {
                fsegs.push_back(ab[k]);
                fsegs.push_back(ab[k] + mh[k]);
                fsegs.push_back(ab[k] + mh[k]);
                fsegs.push_back(ae[k]);
            }
            if ((r2 = seg_sort(c, s->keys.p, s->keys_tmp.p, fsegs, s->seg.p))) return r2;
            k_keys_to_cells<<<gcell, kT, 0, c->stream>>>(L, s->keys.p, s->cells.p);
            k_fill<<<blocks_for(2 * na), kT, 0, c->stream>>>(L, C, s->cells.p, S, s->stripe_of.p);
            k_stripe_minmax<<<gcell, kT, 0, c->stream>>>(L, C, s->cells.p, S, s->stripe_of.p);
            k_new_pos<<<gcell, kT, 0, c->stream>>>(L, C, s->cells.p, S, s->stripe_of.p);
            c->launches += 4;
            KTG_CUDA(c, cudaGetLastError());
            // children
            std::vector<double> halfbox(8 * na);
            KTG_CUDA(c, cudaMemcpyAsync(halfbox.data(), s->half_box.p, sizeof(double) * 8 * na,
                                        cudaMemcpyDeviceToHost, c->stream));
            KTG_CUDA(c, cudaStreamSynchronize(c->stream));
            hb.clear();
            he.clear();
            hv.clear();
            hbox.clear();
            hroom.clear();
            for (int32_t k = 0; k < na; ++k) {
                for (int side = 0; side < 2; ++side) {
                    hb.push_back(side ? ab[k] + mh[k] : ab[k]);
                    he.push_back(side ? ae[k] : ab[k] + mh[k]);
                    hv.push_back(av[k] ? 0 : 1);
                    for (int q = 0; q < 4; ++q) hbox.push_back(halfbox[8 * k + 4 * side + q]);
                    hroom.push_back(aroom[k]);
                }
            }
        }
        batch.clear();
        batch_reach.clear();
        return refresh();
    };

    for (const auto &cl : HG.clusters(occ)) {
        auto bins = HG.grown(cl, occ);
        bool clash = false;
        const auto rb = reach(bins);
        for (const auto &t : batch_reach)
            if (touches(t, rb)) clash = true;
        if (clash) {
            if ((rc = run_batch())) return rc;
            bins = HG.grown(cl, occ);
        }
        batch.push_back(bins);
        batch_reach.push_back(reach(bins));
    }
    if ((rc = run_batch())) return rc;
    if (n > 0) {
        k_clamp_die<<<blocks_for(n), kT, 0, c->stream>>>(C, n, s->die[0], s->die[1], s->die[2],
                                                         s->die[3]);
        ++c->launches;
    }
    KTG_CUDA(c, cudaGetLastError());
    return KTG_OK;
}

}  // namespace ktg
