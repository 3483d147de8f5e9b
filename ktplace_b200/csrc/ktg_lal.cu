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
#include <chrono>
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

int blocks_for(int64_t items, int threads = kT) {
    return static_cast<int>(std::max<int64_t>(1, (items + threads - 1) / threads));
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

// Chunks [b, e) of at most kSortSmall keys, one per block, sorted in shared
// memory; the chunk list holds (b, e) pairs.
__global__ void __launch_bounds__(kT) k_sort_chunks_multi(Key *keys, const int64_t *chunks) {
    __shared__ Key s[kSortSmall];
    const int64_t c0 = chunks[2 * blockIdx.x], c1 = chunks[2 * blockIdx.x + 1];
    const int len = static_cast<int>(c1 - c0);
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

// Segment of global position g among the segments whose lengths prefix
// `pref` (nseg + 1 entries): the last s with pref[s] <= g.
__device__ __forceinline__ int seg_of(const int64_t *pref, int nseg, int64_t g) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pref[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// One merge pass over every long segment at once: runs of `run` keys merged
// pairwise (stable); a segment no longer than `run` is copied across.
__global__ void k_merge_pass_multi(const Key *src, Key *dst, const int64_t *segs,
                                   const int64_t *pref, int nseg, int64_t run) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= pref[nseg]) return;
    const int sg = seg_of(pref, nseg, g);
    const int64_t b = segs[2 * sg], len = segs[2 * sg + 1] - b, r = g - pref[sg];
    if (run >= len) {
        dst[b + r] = src[b + r];
        return;
    }
    const int64_t a0 = (r / (2 * run)) * 2 * run;
    const int64_t a1 = min(a0 + run, len);
    const int64_t b1 = min(a0 + 2 * run, len);
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

__global__ void k_copy_multi(const Key *src, Key *dst, const int64_t *segs, const int64_t *pref,
                             int nseg) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= pref[nseg]) return;
    const int sg = seg_of(pref, nseg, g);
    const int64_t q = segs[2 * sg] + g - pref[sg];
    dst[q] = src[q];
}

// Sorts keys[b, e) of every segment (host list of (b, e) pairs): segments of
// up to kSortSmall keys one block each; longer ones in chunks, then merge
// passes over all of them together. `dseg` holds the device descriptors.
int seg_sort(ktg_ctx *c, Key *keys, Key *tmp, const std::vector<int64_t> &hseg,
             DevBuf<int64_t> &dseg) {
    const int nseg = static_cast<int>(hseg.size() / 2);
    if (nseg == 0) return KTG_OK;
    std::vector<int64_t> small, chunks, large, pref(1, 0);
    int64_t maxlen = 0;
    for (int s = 0; s < nseg; ++s) {
        const int64_t b = hseg[2 * s], e = hseg[2 * s + 1];
        if (e - b <= 1) continue;
        if (e - b <= kSortSmall) {
            small.push_back(b);
            small.push_back(e);
            continue;
        }
        for (int64_t q = b; q < e; q += kSortSmall) {
            chunks.push_back(q);
            chunks.push_back(std::min(e, q + kSortSmall));
        }
        large.push_back(b);
        large.push_back(e);
        pref.push_back(pref.back() + (e - b));
        maxlen = std::max(maxlen, e - b);
    }
    // descriptors: small pairs, chunk pairs, long segments, their prefix
    std::vector<int64_t> all;
    all.reserve(small.size() + chunks.size() + large.size() + pref.size());
    all.insert(all.end(), small.begin(), small.end());
    all.insert(all.end(), chunks.begin(), chunks.end());
    all.insert(all.end(), large.begin(), large.end());
    all.insert(all.end(), pref.begin(), pref.end());
    int rc;
    if ((rc = dseg.ensure(c, static_cast<int64_t>(all.size()) + 1))) return rc;
    KTG_CUDA(c, cudaMemcpyAsync(dseg.p, all.data(), sizeof(int64_t) * all.size(),
                                cudaMemcpyHostToDevice, c->stream));
    const int64_t *d_small = dseg.p;
    const int64_t *d_chunks = d_small + small.size();
    const int64_t *d_large = d_chunks + chunks.size();
    const int64_t *d_pref = d_large + large.size();
    if (!small.empty()) {
        k_sort_small<<<static_cast<int>(small.size() / 2), kT, 0, c->stream>>>(
            keys, d_small, static_cast<int>(small.size() / 2));
        ++c->launches;
    }
    if (!large.empty()) {
        const int nl = static_cast<int>(large.size() / 2);
        const int64_t total = pref.back();
        k_sort_chunks_multi<<<static_cast<int>(chunks.size() / 2), kT, 0, c->stream>>>(keys,
                                                                                     d_chunks);
        ++c->launches;
        Key *src = keys, *dst = tmp;
        for (int64_t run = kSortSmall; run < maxlen; run *= 2) {
            k_merge_pass_multi<<<blocks_for(total), kT, 0, c->stream>>>(src, dst, d_large, d_pref,
                                                                       nl, run);
            ++c->launches;
            std::swap(src, dst);
        }
        if (src != keys) {
            k_copy_multi<<<blocks_for(total), kT, 0, c->stream>>>(src, keys, d_large, d_pref, nl);
            ++c->launches;
        }
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
    int32_t lo = r0, hi = F.R;  // first row from r0 with y start >= uy
    while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (F.rowy[2 * mid] < box[3]) lo = mid + 1;
        else hi = mid;
    }
    const int32_t r1 = lo;
    const int64_t sp = F.rowspan[r1] - F.rowspan[r0];
    steps = vertical ? 2 * sp : 0;
    edges = (vertical ? 2 * sp : 2 * static_cast<int64_t>(r1 - r0)) + 2;
}

// Vertical profile steps of `box` (unsorted), handed to sink(at, dh) in
// row and span order; returns the count.
// First span of row r ending after x (spans of a row ascend and are
// disjoint, FreeSpace::build).
__device__ __forceinline__ int64_t first_span(const Free &F, int32_t r, double x) {
    int64_t lo = F.rowspan[r], hi = F.rowspan[r + 1];
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (F.spans[2 * mid + 1] > x) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// Rows [r0, r1) a box's row loops visit (rows sorted by y start).
__device__ __forceinline__ void box_rows(const Free &F, const double *box, int32_t &r0,
                                         int32_t &r1) {
    r0 = first_row(F, box[1]);
    int32_t lo = r0, hi = F.R;
    while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (F.rowy[2 * mid] < box[3]) lo = mid + 1;
        else hi = mid;
    }
    r1 = lo;
}

// Steps of row r inside box (emit_steps restricted to one row), written
// through sink(k + i, x, dh); returns their count.
template <typename Sink>
__device__ __forceinline__ int64_t row_steps(const Free &F, int32_t r, const double *box, Sink sink,
                                             int64_t k) {
    const double lx = box[0], ly = box[1], ux = box[2], uy = box[3];
    const double h = ref_min(uy, F.rowy[2 * r + 1]) - ref_max(ly, F.rowy[2 * r]);
    if (!(h > 0.0)) return 0;
    const int64_t end = F.rowspan[r + 1];
    int64_t c = 0;
    for (int64_t s = first_span(F, r, lx); s < end && F.spans[2 * s] < ux; ++s) {
        const double a = ref_max(F.spans[2 * s], lx);
        const double z = ref_min(F.spans[2 * s + 1], ux);
        if (z > a) {
            sink(k + c, a, h);
            sink(k + c + 1, z, -h);
            c += 2;
        }
    }
    return c;
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

// Builds the profile of `box` into e/p from its sorted steps (vertical;
// step(k, at, dh) reads the k-th) or the rows (horizontal); returns the
// number of edges.
template <typename Step>
__device__ int64_t build_profile_from(const Free &F, const double *box, bool vertical, Step step,
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
            double at, dh;
            step(k, at, dh);
            extend(at, height * (at - e[n - 1]));
            height += dh;
        }
    } else {
        for (int32_t r = first_row(F, ly); r < F.R && F.rowy[2 * r] < uy; ++r) {
            const double a = ref_max(lo, F.rowy[2 * r]);
            const double z = ref_min(hi, F.rowy[2 * r + 1]);
            if (z > a) {
                extend(a, 0.0);
                // Row::getLength(b.getX()); spans outside [lx, ux] add +0.0
                double total = 0.0;
                const int64_t end = F.rowspan[r + 1];
                for (int64_t s = first_span(F, r, lx); s < end && F.spans[2 * s] < ux; ++s)
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

// getStripes (simpl_lal.cc:266-312) for one half box, then the stable sort
// of nonlinearScale (:325-328) by distance from the cutline, farthest first.
// The reference inserts each midpoint split into its cut list and steps on;
// that visits the intervals depth first, which a small stack does here with
// the same operations (room.getBetween(a, b) = before(b) - before(a), each
// before() computed once). The stripes come out in ascending position, so
// their distance from the cut is monotone: below the cut the stable
// descending order is the order itself, above it the runs of equal distance
// in reverse with each run kept in order. `cuts` is scratch of `cap` doubles;
// the stripes' spans and capacities go to sa/sb/scap. Returns the number of
// stripes, or -1 when `cap` (or the split depth) is exceeded.
__device__ int64_t make_stripes(const Prof &room, const double *box, bool v, double cell_area,
                                double region_room, double frac, double limit_density,
                                const double *obst, int32_t K, double cutline, bool below,
                                double *cuts, int64_t cap, double *sa, double *sb, double *scap) {
    constexpr int kLocalCuts = 64;
    constexpr int kDepth = 64;
    const double lo = v ? box[0] : box[1], hi = v ? box[2] : box[3];
    double lc[kLocalCuts];  // small cut lists are sorted in (L1-resident) local memory
    int64_t nc = 0;
    bool local = true;
    auto put = [&](double x) {
        if (local && nc < kLocalCuts) {
            lc[nc++] = x;
            return;
        }
        if (local) {
            for (int64_t i = 0; i < nc; ++i) cuts[i] = lc[i];
            local = false;
        }
        cuts[nc++] = x;
    };
    put(lo);
    put(hi);
    for (int32_t o = 0; o < K; ++o) {
        const double *ob = obst + 4 * o;
        if (ob[2] <= box[0] || ob[0] >= box[2] || ob[3] <= box[1] || ob[1] >= box[3]) continue;
        const double e0 = v ? ob[0] : ob[1], e1 = v ? ob[2] : ob[3];
        if (nc + 2 > cap) return -1;
        if (e0 > lo && e0 < hi) put(e0);
        if (e1 > lo && e1 < hi) put(e1);
    }
    double *c = local ? lc : cuts;
    for (int64_t i = 1; i < nc; ++i) {  // insertion sort (stable)
        const double t = c[i];
        int64_t j = i - 1;
        while (j >= 0 && t < c[j]) {
            c[j + 1] = c[j];
            --j;
        }
        c[j + 1] = t;
    }
    int64_t u = 0;
    for (int64_t i = 0; i < nc; ++i)
        if (u == 0 || !(c[u - 1] == c[i])) c[u++] = c[i];
    nc = u;
    const double limit = frac * (region_room > 0.0 ? region_room : room.total());
    const double fill = room.total() > 0.0 ? ref_min(limit_density, cell_area / room.total())
                                           : limit_density;
    int64_t ns = 0;
    double a = c[0], ba = room.before(a);
    double stk[kDepth], stkb[kDepth];
    for (int64_t i = 1; i < nc; ++i) {
        int top = 0;
        stk[top] = c[i];
        stkb[top] = room.before(c[i]);
        ++top;
        while (top > 0) {
            const double b = stk[top - 1], bb = stkb[top - 1];
            const double here = bb - ba;
            const double mid = room.coordinate_at(ba + 0.5 * here);
            if (here > limit && mid > a && mid < b) {
                if (top == kDepth || ns + top + 1 > cap) return -1;
                stk[top] = mid;
                stkb[top] = room.before(mid);
                ++top;
            } else {
                if (ns >= cap) return -1;
                sa[ns] = a;
                sb[ns] = b;
                scap[ns] = fill * here;
                ++ns;
                --top;
                a = b;
                ba = bb;
            }
        }
    }
    if (!below) {
        auto swap_at = [&](int64_t i, int64_t j) {
            double t = sa[i]; sa[i] = sa[j]; sa[j] = t;
            t = sb[i]; sb[i] = sb[j]; sb[j] = t;
            t = scap[i]; scap[i] = scap[j]; scap[j] = t;
        };
        for (int64_t i = 0, j = ns - 1; i < j; ++i, --j) swap_at(i, j);
        for (int64_t r = 0; r < ns;) {  // restore the original order inside each run
            const double f = 0.5 * (sa[r] + sb[r]) - cutline;
            int64_t e = r + 1;
            while (e < ns && 0.5 * (sa[e] + sb[e]) - cutline == f) ++e;
            for (int64_t i = r, j = e - 1; i < j; ++i, --j) swap_at(i, j);
            r = e;
        }
    }
    return ns;
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
// ---- exact area sums ------------------------------------------------------------
//
// When every cell area is a multiple of 2^-q and the total times 2^q stays
// below 2^52, every partial sum the reference forms (cellArea, lowArea, a
// stripe's used area) is exact in double, whatever the order. The sums are
// then read off an integer prefix over the positions: pre[p] = fixed-point
// area of positions [0, p).

constexpr int kScanTile = 2048;  // positions per tile: kT threads x 8

__device__ __forceinline__ long long area_fx(const double *area, int32_t i, double scale) {
    return __double2ll_rn(area[i] * scale);
}

__device__ __forceinline__ long long warp_incl64(long long v) {
    const int lane = threadIdx.x & 31;
    for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive block scan of one value per thread (blockDim.x == kT); returns
// the exclusive prefix and sets `total`.
__device__ long long block_excl64(long long v, long long &total) {
    __shared__ long long ws[kT / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const long long inc = warp_incl64(v);
    if (lane == 31) ws[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        long long w = lane < kT / 32 ? ws[lane] : 0;
        w = warp_incl64(w);
        if (lane < kT / 32) ws[lane] = w;
    }
    __syncthreads();
    const long long out = inc - v + (wid > 0 ? ws[wid - 1] : 0);
    total = ws[kT / 32 - 1];
    __syncthreads();
    return out;
}

__global__ void __launch_bounds__(kT) k_fx_tile_sums(const int32_t *cells, const double *area,
                                                     int32_t n, double scale, long long *tile) {
    const int32_t base = blockIdx.x * kScanTile;
    long long v = 0;
    for (int k = threadIdx.x; k < kScanTile; k += kT)
        if (base + k < n) v += area_fx(area, cells[base + k], scale);
    long long total;
    block_excl64(v, total);
    if (threadIdx.x == 0) tile[blockIdx.x] = total;
}

// Exclusive scan of the tile sums in place (one block).
__global__ void __launch_bounds__(kT) k_fx_tile_scan(long long *tile, int32_t ntiles) {
    const int per = (ntiles + kT - 1) / kT;
    const int beg = threadIdx.x * per, end = min(beg + per, ntiles);
    long long v = 0;
    for (int i = beg; i < end; ++i) v += tile[i];
    long long total;
    long long run = block_excl64(v, total);
    for (int i = beg; i < end; ++i) {
        const long long t = tile[i];
        tile[i] = run;
        run += t;
    }
}

// pre[p + 1] = fixed-point area of positions [0, p]; pre[0] = 0.
__global__ void __launch_bounds__(kT) k_fx_prefix(const int32_t *cells, const double *area,
                                                  int32_t n, double scale, const long long *tile,
                                                  long long *pre) {
    const int32_t base = blockIdx.x * kScanTile + threadIdx.x * (kScanTile / kT);
    long long v[kScanTile / kT];
    long long sum = 0;
#pragma unroll
    for (int k = 0; k < kScanTile / kT; ++k) {
        v[k] = base + k < n ? area_fx(area, cells[base + k], scale) : 0;
        sum += v[k];
    }
    long long total;
    long long run = block_excl64(sum, total) + tile[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanTile / kT; ++k) {
        run += v[k];
        if (base + k < n) pre[base + k + 1] = run;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) pre[0] = 0;
}

// Median split from the prefix: the least m >= 1 with 2 * low(m) >= total,
// at most size - 1 (the loop of split, simpl_lal.cc:230-233).
__device__ __forceinline__ int32_t median_fx(const long long *pre, int32_t b, int32_t size) {
    if (size <= 1) return 0;
    const long long tot = pre[b + size] - pre[b];
    int32_t lo = 1, hi = size - 1;  // answer in [lo, hi]
    while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (2 * (pre[b + mid] - pre[b]) >= tot) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// One thread per block: areas and median in the reference's order (or from
// the exact prefix when `pre` is set), and the block profile's bound.
__global__ void k_block_split(Level L, CellsDev C, Free F, const int32_t *cells,
                              const long long *pre, double inv_scale) {
    const int32_t blk = blockIdx.x * blockDim.x + threadIdx.x;
    if (blk >= L.na) return;
    const int32_t b = L.b[blk], e = L.e[blk];
    const int32_t size = e - b;
    double cell_area = 0.0, low = 0.0, high = 0.0;
    int32_t m = 0;
    if (pre) {
        m = median_fx(pre, b, size);
        cell_area = static_cast<double>(pre[e] - pre[b]) * inv_scale;
        low = static_cast<double>(pre[b + m] - pre[b]) * inv_scale;
        high = static_cast<double>(pre[e] - pre[b + m]) * inv_scale;
    } else {
        for (int32_t p = b; p < e; ++p) cell_area += C.area[cells[p]];
        while (m + 1 < size && (m == 0 || low < 0.5 * cell_area)) low += C.area[cells[b + m++]];
        for (int32_t p = b + m; p < e; ++p) high += C.area[cells[p]];
    }
    L.m[blk] = m;
    L.low_area[blk] = low;
    L.high_area[blk] = high;
    L.cut[blk] = cell_area;  // kept until the cutline replaces it
    int64_t st, ed;
    profile_bound(F, L.box + 4 * blk, L.vert[blk] != 0, st, ed);
    L.bound[2 * blk] = st;
    L.bound[2 * blk + 1] = ed;
}

// One thread per block: profile, cutline, half boxes, half bounds.
struct Stripes {
    int64_t *off;    // [2 na] first stripe of the half (into the arrays below)
    int32_t *count;  // [2 na]
    double *a, *b, *cap, *used;
    unsigned long long *lo, *hi;
};

// ---- one CTA per block (or half) for the level-by-level path ------------------------
//
// Blocks too large for the one-CTA subtree have die-sized boxes: their row
// loops are split over the CTA's threads and the profile is built by thread 0
// from chunks staged in shared memory (the order of its sums is the
// reference's).

constexpr int kStage = 1024;

// Builds the profile of `box` into e/p (global). Returns the edge count on
// thread 0.
__device__ int64_t cta_build_profile(const Free &F, const double *box, bool v, const Key *steps,
                                     int64_t nsteps, double *e, double *p, double *stage) {
    const double lx = box[0], ly = box[1], ux = box[2], uy = box[3];
    const double lo = v ? lx : ly, hi = v ? ux : uy;
    const int tid = threadIdx.x, nt = blockDim.x;
    int64_t n = 1;
    double elast = lo, plast = 0.0, height = 0.0;
    auto extend = [&](double to, double area) {
        if (to > elast) {
            plast = plast + area;
            elast = to;
            e[n] = to;
            p[n] = plast;
            ++n;
        }
    };
    if (tid == 0) {
        e[0] = lo;
        p[0] = 0.0;
    }
    if (v) {
        // chunk c + 1 is loaded into registers while thread 0 walks chunk c
        constexpr int kPer = kStage / kT;
        Key nxt[kPer];
        auto fetch = [&](int64_t c0) {
#pragma unroll
            for (int u = 0; u < kPer; ++u) {
                const int64_t k = c0 + u * nt + tid;
                nxt[u] = k < nsteps ? steps[k] : Key{0ull, 0ull};
            }
        };
        fetch(0);
        for (int64_t c0 = 0; c0 < nsteps; c0 += kStage) {
            const int cnt = static_cast<int>(nsteps - c0 < kStage ? nsteps - c0 : kStage);
            __syncthreads();  // the previous chunk is consumed
#pragma unroll
            for (int u = 0; u < kPer; ++u) {
                const int i = u * nt + tid;
                if (i < cnt) {
                    stage[2 * i] = unord(nxt[u].a);
                    stage[2 * i + 1] = unord(nxt[u].b);
                }
            }
            __syncthreads();
            fetch(c0 + kStage);
            if (tid == 0)
                for (int i = 0; i < cnt; ++i) {
                    const double at = stage[2 * i], dh = stage[2 * i + 1];
                    extend(at, height * (at - elast));
                    height += dh;
                }
        }
        __syncthreads();
    } else {
        int32_t r0, r1;
        box_rows(F, box, r0, r1);
        for (int32_t c0 = r0; c0 < r1; c0 += kStage) {
            const int cnt = min(kStage, r1 - c0);
            for (int i = tid; i < cnt; i += nt) {  // Row::getLength(b.getX())
                const int32_t r = c0 + i;
                double total = 0.0;
                const int64_t end = F.rowspan[r + 1];
                for (int64_t q = first_span(F, r, lx); q < end && F.spans[2 * q] < ux; ++q)
                    total += ref_max(0.0, ref_min(ux, F.spans[2 * q + 1]) - ref_max(lx, F.spans[2 * q]));
                stage[i] = total;
            }
            __syncthreads();
            if (tid == 0)
                for (int i = 0; i < cnt; ++i) {
                    const int32_t r = c0 + i;
                    const double a = ref_max(lo, F.rowy[2 * r]);
                    const double z = ref_min(hi, F.rowy[2 * r + 1]);
                    if (z > a) {
                        extend(a, 0.0);
                        extend(z, stage[i] * (z - a));
                    }
                }
            __syncthreads();
        }
    }
    if (tid == 0) {
        extend(hi, 0.0);
        if (n == 1) {
            e[1] = hi;
            p[1] = 0.0;
            n = 2;
        }
    }
    return n;
}

// Profile steps of each block (half = 0) or half box (half = 1), one CTA
// each, rows split over the threads.
__global__ void __launch_bounds__(kT) k_steps_cta(Level L, Free F, int half, const int64_t *soff,
                                                  Key *steps, int64_t *nsteps) {
    const int item = blockIdx.x;
    const int blk = half ? item >> 1 : item;
    const double *box = half ? L.half_box + 4 * item : L.box + 4 * item;
    if (!L.vert[blk]) {
        if (threadIdx.x == 0) nsteps[item] = 0;
        return;
    }
    int32_t r0, r1;
    box_rows(F, box, r0, r1);
    long long c = 0;
    for (int32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x)
        c += row_steps(F, r, box, [](int64_t, double, double) {}, 0);
    long long total;
    int64_t k = block_excl64(c, total);
    Key *out = steps + soff[item];
    auto sink = [&](int64_t q, double x, double dh) { out[q] = Key{ord(x), ord(dh)}; };
    for (int32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) k += row_steps(F, r, box, sink, k);
    if (threadIdx.x == 0) nsteps[item] = total;
}

// One CTA per block: profile, cutline, half boxes, half bounds.
__global__ void __launch_bounds__(kT) k_block_cut_cta(Level L, Free F, const int64_t *soff,
                                                      const Key *steps, const int64_t *nsteps,
                                                      const int64_t *eoff, double *pe, double *pp,
                                                      int64_t *hbound) {
    __shared__ double stage[2 * kStage];
    const int blk = blockIdx.x;
    const bool v = L.vert[blk] != 0;
    const double *box = L.box + 4 * blk;
    double *e = pe + eoff[blk], *p = pp + eoff[blk];
    const int64_t n = cta_build_profile(F, box, v, steps + soff[blk], nsteps[blk], e, p, stage);
    if (threadIdx.x == 0) {
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
    }
    __syncthreads();
    for (int side = 0; side < 2; ++side) {
        const double *bx = L.half_box + 8 * blk + 4 * side;
        long long k = 0;  // obstacles overlapping the half box
        for (int32_t o = threadIdx.x; o < F.K; o += blockDim.x) {
            const double *ob = F.obst + 4 * o;
            if (ob[2] <= bx[0] || ob[0] >= bx[2] || ob[3] <= bx[1] || ob[1] >= bx[3]) continue;
            ++k;
        }
        long long total;
        block_excl64(k, total);
        if (threadIdx.x == 0) {
            int64_t st, ed;
            profile_bound(F, bx, v, st, ed);
            hbound[4 * blk + 2 * side] = st;
            hbound[4 * blk + 2 * side + 1] = ed + 2 * total + 2;  // profile edges, obstacle cuts
        }
    }
}

// One CTA per half: profile, stripes (getStripes), fill state. A profile of
// up to kProfSmem edges is copied to shared memory before the stripe loop,
// whose profile lookups are then shared-memory binary searches.
constexpr int kProfSmem = 6144;
constexpr size_t kHalfStripesSmem = sizeof(double) * 2 * kProfSmem;

__global__ void __launch_bounds__(kT) k_half_stripes_cta(Level L, Free F, const int64_t *soff,
                                                         const Key *steps, const int64_t *nsteps,
                                                         const int64_t *eoff, double *pe, double *pp,
                                                         const int64_t *cap_over, double frac,
                                                         double limit_density, Stripes S,
                                                         int *status) {
    __shared__ double stage[2 * kStage];
    __shared__ long long s_ns, s_n;
    extern __shared__ double prof[];  // [2 * kProfSmem]
    const int h = blockIdx.x;
    const int blk = h >> 1, side = h & 1;
    const bool v = L.vert[blk] != 0;
    const double *box = L.half_box + 4 * h;
    double *e = pe + eoff[h], *p = pp + eoff[h];
    const int64_t n0 = cta_build_profile(F, box, v, steps + soff[h], nsteps[h], e, p, stage);
    if (threadIdx.x == 0) s_n = n0;
    __syncthreads();
    const int64_t n = s_n;
    const bool local = n <= kProfSmem;
    if (local) {
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            prof[i] = e[i];
            prof[kProfSmem + i] = p[i];
        }
        __syncthreads();
    }
    const int64_t so = S.off[h];
    if (threadIdx.x == 0) {
        const Prof room{local ? prof : e, local ? prof + kProfSmem : p, n};
        const double cell_area = side ? L.high_area[blk] : L.low_area[blk];
        // cuts live after the profile in the global scratch
        int64_t ns = make_stripes(room, box, v, cell_area, L.room[blk], frac, limit_density,
                                  F.obst, F.K, L.cut[blk], side == 0, p + n, cap_over[h],
                                  S.a + so, S.b + so, S.cap + so);
        if (ns < 0) {
            atomicCAS(status, kStatusOk, kStatusCapacity);
            ns = 0;
        }
        S.count[h] = static_cast<int32_t>(ns);
        s_ns = ns;
    }
    __syncthreads();
    for (int64_t q = threadIdx.x; q < s_ns; q += blockDim.x) {
        S.used[so + q] = 0.0;
        S.lo[so + q] = ~0ull;
        S.hi[so + q] = 0ull;
    }
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

// Greedy fill from the exact prefix (fill order): stripe s of a half takes
// positions [start_s, start_{s+1}), start_{s+1} the least position whose
// preceding area in the stripe reaches its capacity. One CTA per half; each
// start is found by rounds of kT-way probing of the (monotone) prefix. The
// starts go to `sbeg`.
__global__ void __launch_bounds__(kT) k_fill_fx(Level L, Stripes S, const long long *pre,
                                                double inv_scale, int32_t *sbeg) {
    __shared__ int32_t s_lo, s_hi, s_first;
    const int32_t h = blockIdx.x;
    const int32_t blk = h >> 1;
    const int32_t b = L.b[blk], e = L.e[blk], mid = b + L.m[blk];
    const int32_t p0 = (h & 1) ? mid : b, p1 = (h & 1) ? e : mid;
    const int64_t so = S.off[h];
    const int32_t ns = S.count[h];
    int32_t at = p0;
    for (int32_t s = 0; s < ns; ++s) {
        if (threadIdx.x == 0) sbeg[so + s] = at;
        if (s + 1 == ns) break;
        const double cap = S.cap[so + s];
        const long long base = pre[at];
        // least k in [at, p1] with used(k) >= cap, p1 counting as true
        auto hit = [&](int32_t k) {
            return k >= p1 || static_cast<double>(pre[k] - base) * inv_scale >= cap;
        };
        int32_t lo = at, hi = p1;
        while (hi - lo + 1 > kT) {
            const int32_t step = (hi - lo + kT) / kT;  // ceil((hi - lo + 1) / kT)
            if (threadIdx.x == 0) s_first = kT;
            __syncthreads();
            const int32_t k = min(hi, lo + (threadIdx.x + 1) * step - 1);
            if (hit(k)) atomicMin(&s_first, static_cast<int32_t>(threadIdx.x));
            __syncthreads();
            const int32_t f = s_first;
            const int32_t nlo = f == 0 ? lo : min(hi, lo + f * step - 1) + 1;
            const int32_t nhi = min(hi, lo + (f + 1) * step - 1);
            __syncthreads();
            lo = nlo;
            hi = nhi;
        }
        if (threadIdx.x == 0) s_first = hi;
        __syncthreads();
        if (lo + static_cast<int32_t>(threadIdx.x) <= hi && hit(lo + threadIdx.x))
            atomicMin(&s_first, lo + static_cast<int32_t>(threadIdx.x));
        __syncthreads();
        at = s_first;
        __syncthreads();
    }
}

// Stripe of every position: the last stripe of its half starting at or
// before it.
__global__ void k_assign_fx(Level L, const int32_t *cells, Stripes S, const int32_t *sbeg,
                            int32_t *stripe_of) {
    for (int32_t blk = blockIdx.y; blk < L.na; blk += gridDim.y) {
        const int32_t b = L.b[blk], e = L.e[blk], mid = b + L.m[blk];
        for (int32_t p = b + blockIdx.x * blockDim.x + threadIdx.x; p < e; p += gridDim.x * blockDim.x) {
            const int32_t h = 2 * blk + (p < mid ? 0 : 1);
            const int64_t so = S.off[h];
            const int32_t ns = S.count[h];
            int32_t s = -1;
            if (ns > 0) {
                int32_t lo = 0, hi = ns - 1;  // last s with sbeg[s] <= p (sbeg[0] <= p)
                while (lo < hi) {
                    const int32_t k = (lo + hi + 1) >> 1;
                    if (sbeg[so + k] <= p) lo = k;
                    else hi = k - 1;
                }
                s = static_cast<int32_t>(so + lo);
            }
            stripe_of[cells[p]] = s;
        }
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

// ---- small blocks: one CTA finishes a block's whole subtree ------------------------
//
// A block of at most kSub cells is handed to one CTA, which runs every
// remaining level of its bisection out of shared memory: the cells' ids,
// positions, sizes and areas, the CTA-wide sort buffer (three key words per
// entry, compared as (k2, k0, k1)) and the per-level scans. The level's
// sub-blocks, their profiles and stripes live in a per-CTA slice of global
// scratch. A block whose needs exceed a capacity (sort buffer, profile or
// stripe slots, sub-blocks per level, local obstacles) is left untouched
// and flagged; the caller runs it level by level instead.

constexpr int kSub = 2048;
constexpr int kSubThreads = 512;
constexpr int kSortCap = 4096;      // entries of the sort buffer (steps and profiles)
constexpr int kMaxSub = 1024;       // sub-blocks of one level
constexpr int kObstLocal = 256;     // obstacles overlapping the block
constexpr int64_t kStripeCap = 8192;
constexpr int kRowsLocal = 512;     // free-space rows staged in shared memory
constexpr int kSpansLocal = 1280;   // and their spans
constexpr size_t kSubSmem = sizeof(unsigned long long) * 2 * kSortCap +
                            sizeof(uint32_t) * kSortCap + sizeof(long long) * (kSub + 2) +
                            sizeof(double) * (3 * kSub + 4 * kObstLocal) +
                            sizeof(double) * (2 * kRowsLocal + 2 * kSpansLocal) +
                            sizeof(int64_t) * (kRowsLocal + 2) +
                            sizeof(int32_t) * (3 * kSub + 2 * kMaxSub + 2) + sizeof(int16_t) * kSub;

struct SubTask {
    double box[4];
    double room;
    int32_t b, e, level, vert;
};

struct SubDesc {
    double box[4];
    double hbox[8];
    double cell_area, low_area, high_area, cut;
    int32_t b, e, level, vert, m, act, rank;
    int32_t soff, scnt, slen;                     // block profile region in the sort buffer
    int32_t hsoff[2], hscnt[2], hslen[2];         // the halves' regions
    int32_t stoff[2], stcap[2], stcnt[2];         // the halves' stripes
};

struct SubArgs {
    const SubTask *tasks;
    int32_t ntasks;
    int32_t *fail;           // [ntasks] 1: left for the level-by-level path
    const int32_t *cells;    // position -> cell id
    CellsDev C;
    Free F;
    SubDesc *desc;           // [grid * 2 * kMaxSub]
    double *strp;            // [grid * 4 * kStripeCap] cuts, start, end, capacity
    unsigned long long *strlh;  // [grid * 2 * kStripeCap] lowest / highest centre
    int32_t max_level, min_cells, stripe_extra;
    double frac, limit_density;
    int32_t exact;           // areas sum exactly: prefix sums and binary searches
    double scale, inv_scale; // 2^q, 2^-q
};

__device__ __forceinline__ bool sub_less(uint32_t a2, unsigned long long a0, unsigned long long a1,
                                         uint32_t b2, unsigned long long b0, unsigned long long b1) {
    return a2 < b2 || (a2 == b2 && (a0 < b0 || (a0 == b0 && a1 < b1)));
}

// In-place sort of entries [b, b + n) by `nthreads` cooperating threads
// (index `me`), for any n: every merge of two sorted halves starts with the
// mirrored comparators (i, k - 1 - i) and continues with half-cleaners, all
// ascending, so positions past n act as +inf and their comparators are
// skipped. `sync` separates the steps (a warp or the whole block).
template <typename Sync>
__device__ void net_sort(unsigned long long *k0, unsigned long long *k1, uint32_t *k2, int b, int n,
                         int me, int nthreads, Sync sync) {
    if (n <= 1) return;
    int P = 1;
    while (P < n) P <<= 1;
    auto cas = [&](int i, int q) {
        const uint32_t a2 = k2[b + i], b2 = k2[b + q];
        const unsigned long long a0 = k0[b + i], b0 = k0[b + q], a1 = k1[b + i], b1 = k1[b + q];
        if (sub_less(b2, b0, b1, a2, a0, a1)) {
            k2[b + i] = b2; k0[b + i] = b0; k1[b + i] = b1;
            k2[b + q] = a2; k0[b + q] = a0; k1[b + q] = a1;
        }
    };
    for (int k = 2; k <= P; k <<= 1) {
        const int h = k >> 1;
        for (int t = me; t < (P >> 1); t += nthreads) {
            const int base = (t / h) * k, off = t % h;
            const int q = base + k - 1 - off;
            if (q < n) cas(base + off, q);
        }
        sync();
        for (int j = k >> 2; j > 0; j >>= 1) {
            for (int t = me; t < (P >> 1); t += nthreads) {
                const int i = 2 * j * (t / j) + (t % j);
                if (i + j < n) cas(i, i + j);
            }
            sync();
        }
    }
}

__device__ __forceinline__ void named_barrier(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Sorts each segment [b, e) = seg(g) of g < nseg (none longer than maxlen):
// the whole block for one segment, equal groups of warps (each on its own
// named barrier) for a few long ones, else teams of lanes sized to the
// longest segment (one lane for up to 3 keys, up to a warp), each team
// taking segments in turn. Ends with a block barrier.
template <typename Seg>
__device__ void sort_segments(unsigned long long *k0, unsigned long long *k1, uint32_t *k2, int nseg,
                              int maxlen, Seg seg) {
    const int nw = blockDim.x >> 5, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (nseg <= 0 || maxlen <= 1) {
        __syncthreads();
        return;
    }
    if (nseg == 1) {
        int b, e;
        seg(0, b, e);
        net_sort(k0, k1, k2, b, e - b, threadIdx.x, blockDim.x, [] { __syncthreads(); });
    } else if (nseg < 16 && nw / nseg >= 2 && maxlen > 256) {
        const int W = nw / nseg;  // warps per group
        const int g = w / W;
        if (g < nseg) {
            int b, e;
            seg(g, b, e);
            const int me = (w - g * W) * 32 + lane, n = W * 32;
            net_sort(k0, k1, k2, b, e - b, me, n, [g, n] { named_barrier(1 + g, n); });
        }
    } else {
        int T = 1;  // lanes per team: about half the longest segment, at most a warp
        while (T < 32 && 2 * T < maxlen) T <<= 1;
        const int me = threadIdx.x & (T - 1), team = threadIdx.x / T, nteams = blockDim.x / T;
        const unsigned mask = T == 32 ? 0xffffffffu : (((1u << T) - 1u) << (lane & ~(T - 1)));
        for (int g = team; g < nseg; g += nteams) {
            int b, e;
            seg(g, b, e);
            net_sort(k0, k1, k2, b, e - b, me, T, [mask] { __syncwarp(mask); });
        }
    }
    __syncthreads();
}

// Exclusive scan of buf[0, n) in place; returns the total to every thread.
__device__ int32_t cta_scan(int32_t *buf, int n, int32_t *warp_tmp) {
    const int nt = blockDim.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int per = (n + nt - 1) / nt;
    const int beg = min(tid * per, n), end = min(beg + per, n);
    int32_t local = 0;
    for (int i = beg; i < end; ++i) local += buf[i];
    int32_t v = local;
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) warp_tmp[wid] = v;
    __syncthreads();
    const int nw = nt >> 5;
    if (wid == 0) {
        int32_t w = lane < nw ? warp_tmp[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < nw) warp_tmp[lane] = w;
    }
    __syncthreads();
    int32_t run = v - local + (wid > 0 ? warp_tmp[wid - 1] : 0);
    const int32_t total = warp_tmp[nw - 1];
    for (int i = beg; i < end; ++i) {
        const int32_t t = buf[i];
        buf[i] = run;
        run += t;
    }
    __syncthreads();
    return total;
}

// pre[p + 1] = fixed-point area of positions [0, p] (cell at[p], area sa);
// pre[0] = 0.
__device__ void cta_prefix64(const int32_t *at, const double *sa, int n, double scale,
                             long long *pre, long long *w64) {
    const int nt = blockDim.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int per = (n + nt - 1) / nt;
    const int beg = min(tid * per, n), end = min(beg + per, n);
    long long local = 0;
    for (int p = beg; p < end; ++p) local += __double2ll_rn(sa[at[p]] * scale);
    long long v = local;
    for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) w64[wid] = v;
    __syncthreads();
    const int nw = nt >> 5;
    if (wid == 0) {
        long long w = lane < nw ? w64[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const long long t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < nw) w64[lane] = w;
    }
    __syncthreads();
    long long run = v - local + (wid > 0 ? w64[wid - 1] : 0);
    for (int p = beg; p < end; ++p) {
        run += __double2ll_rn(sa[at[p]] * scale);
        pre[p + 1] = run;
    }
    if (tid == 0) pre[0] = 0;
    __syncthreads();
}

// A region of the sort buffer holding a profile: two leading pads, then the
// sorted steps (vertical) or nothing (horizontal); the profile is written
// over it in place (edge n lands at slot n, the step read last sits at slot
// >= n + 1).
__device__ int64_t build_profile_inplace(const Free &F, const double *box, bool v,
                                         unsigned long long *k0, unsigned long long *k1, int o,
                                         int nsteps) {
    double *e = reinterpret_cast<double *>(k0 + o);
    double *p = reinterpret_cast<double *>(k1 + o);
    return build_profile_from(
        F, box, v,
        [&](int64_t k, double &x, double &dh) {
            x = unord(k0[o + 2 + k]);
            dh = unord(k1[o + 2 + k]);
        },
        nsteps, e, p);
}

// A team of T lanes (a power of two up to 32, aligned inside a warp) that
// works on one sub-block: few sub-blocks at a level get wide teams, many get
// one thread each. Row loops are split over the lanes; everything whose
// floating-point order matters runs on lane 0.
struct Team {
    int T, lane, team, nteams;
    unsigned mask;
    __device__ explicit Team(int items) {
        const int per = kSubThreads / max(items, 1);
        T = per >= 32 ? 32 : per >= 16 ? 16 : per >= 8 ? 8 : per >= 4 ? 4 : per >= 2 ? 2 : 1;
        lane = threadIdx.x & (T - 1);
        team = threadIdx.x / T;
        nteams = blockDim.x / T;
        const int wl = threadIdx.x & 31;
        mask = T == 32 ? 0xffffffffu : (((1u << T) - 1u) << (wl & ~(T - 1)));
    }
    template <typename V>
    __device__ V sum(V v) const {
        for (int o = T >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
        return v;
    }
    template <typename V>
    __device__ V excl(V v) const {
        V inc = v;
        for (int o = 1; o < T; o <<= 1) {
            const V t = __shfl_up_sync(mask, inc, o, T);
            if (lane >= o) inc += t;
        }
        return inc - v;
    }
    template <typename V>
    __device__ V bcast(V v) const { return __shfl_sync(mask, v, 0, T); }
    __device__ void sync() const { __syncwarp(mask); }
};

__device__ int32_t team_count_steps(const Team &tm, const Free &F, const double *box) {
    int32_t r0, r1;
    box_rows(F, box, r0, r1);
    int32_t c = 0;
    for (int32_t r = r0 + tm.lane; r < r1; r += tm.T)
        c += static_cast<int32_t>(row_steps(F, r, box, [](int64_t, double, double) {}, 0));
    return tm.sum(c);
}

__device__ int32_t team_count_obstacles(const Team &tm, const Free &F, const double *bx) {
    int32_t k = 0;
    for (int32_t ob = tm.lane; ob < F.K; ob += tm.T) {
        const double *q = F.obst + 4 * ob;
        if (q[2] <= bx[0] || q[0] >= bx[2] || q[3] <= bx[1] || q[1] >= bx[3]) continue;
        ++k;
    }
    return tm.sum(k);
}

// Writes a profile region: pads over [o, o + len), then (vertical) the box's
// steps from o + 2, the rows split over the team (step order inside the
// region does not matter: it is sorted next).
__device__ void team_emit_region(const Team &tm, const Free &F, const double *box, bool v,
                                 uint32_t tag, unsigned long long *k0, unsigned long long *k1,
                                 uint32_t *k2, int o, int len) {
    for (int q = tm.lane; q < len; q += tm.T) {
        k2[o + q] = tag;
        k0[o + q] = 0ull;
        k1[o + q] = 0ull;
    }
    tm.sync();
    if (!v) return;
    int32_t r0, r1;
    box_rows(F, box, r0, r1);
    int32_t c = 0;
    for (int32_t r = r0 + tm.lane; r < r1; r += tm.T)
        c += static_cast<int32_t>(row_steps(F, r, box, [](int64_t, double, double) {}, 0));
    int64_t k = o + 2 + tm.excl(c);
    auto sink = [&](int64_t q, double x, double dh) {
        k0[q] = ord(x);
        k1[q] = ord(dh);
    };
    for (int32_t r = r0 + tm.lane; r < r1; r += tm.T) k += row_steps(F, r, box, sink, k);
    tm.sync();
}

// build_profile_inplace with a team: horizontal boxes get their per-row
// lengths (Row::getLength, each row's spans summed in order by one lane)
// from the lanes first, parked at the top of the region (slots the profile
// reaches only after it has read them); the profile itself is built by lane
// 0. Returns the edge count to every lane.
__device__ int64_t team_build_profile(const Team &tm, const Free &F, const double *box, bool v,
                                      unsigned long long *k0, unsigned long long *k1, int o,
                                      int nsteps, int len) {
    int64_t n = 0;
    if (v) {
        if (tm.lane == 0) n = build_profile_inplace(F, box, v, k0, k1, o, nsteps);
        return tm.bcast(n);
    }
    const double lx = box[0], ly = box[1], ux = box[2], uy = box[3];
    int32_t r0, r1;
    box_rows(F, box, r0, r1);
    const int32_t nr = r1 - r0;
    double *tot = reinterpret_cast<double *>(k1 + o + len - nr);
    for (int32_t i = tm.lane; i < nr; i += tm.T) {
        const int32_t r = r0 + i;
        double total = 0.0;
        const int64_t end = F.rowspan[r + 1];
        for (int64_t s = first_span(F, r, lx); s < end && F.spans[2 * s] < ux; ++s)
            total += ref_max(0.0, ref_min(ux, F.spans[2 * s + 1]) - ref_max(lx, F.spans[2 * s]));
        tot[i] = total;
    }
    tm.sync();
    if (tm.lane == 0) {
        double *e = reinterpret_cast<double *>(k0 + o);
        double *p = reinterpret_cast<double *>(k1 + o);
        n = 1;
        e[0] = ly;
        p[0] = 0.0;
        auto extend = [&](double to, double area) {
            if (to > e[n - 1]) {
                e[n] = to;
                p[n] = p[n - 1] + area;
                ++n;
            }
        };
        for (int32_t i = 0; i < nr; ++i) {
            const int32_t r = r0 + i;
            const double a = ref_max(ly, F.rowy[2 * r]);
            const double z = ref_min(uy, F.rowy[2 * r + 1]);
            if (z > a) {
                const double total = tot[i];
                extend(a, 0.0);
                extend(z, total * (z - a));
            }
        }
        extend(uy, 0.0);
        if (n == 1) {
            e[1] = uy;
            p[1] = 0.0;
            n = 2;
        }
    }
    n = tm.bcast(n);
    tm.sync();
    return n;
}

__global__ void __launch_bounds__(kSubThreads, 1) k_subtree(SubArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned long long *k0 = reinterpret_cast<unsigned long long *>(smem);
    unsigned long long *k1 = k0 + kSortCap;
    long long *pre = reinterpret_cast<long long *>(k1 + kSortCap);  // [kSub + 1]
    double *sx = reinterpret_cast<double *>(pre + kSub + 2);
    double *sy = sx + kSub, *sa = sy + kSub;
    double *obst = sa + kSub;
    double *lrowy = obst + 4 * kObstLocal, *lspans = lrowy + 2 * kRowsLocal;
    int64_t *lrowspan = reinterpret_cast<int64_t *>(lspans + 2 * kSpansLocal);
    uint32_t *k2 = reinterpret_cast<uint32_t *>(lrowspan + kRowsLocal + 2);
    int32_t *gid = reinterpret_cast<int32_t *>(k2 + kSortCap);
    int32_t *at = gid + kSub, *sof = at + kSub, *scan = sof + kSub;
    int16_t *dof = reinterpret_cast<int16_t *>(scan + 2 * kMaxSub + 2);
    __shared__ int32_t warp_tmp[32];
    __shared__ long long w64[32];
    __shared__ int s_fail, s_nobst, s_ncur, s_maxlen, s_maxsteps, s_c1;
    const int tid = threadIdx.x, nt = blockDim.x;
    SubDesc *const cur0 = A.desc + static_cast<size_t>(blockIdx.x) * 2 * kMaxSub;
    double *const scut = A.strp + static_cast<size_t>(blockIdx.x) * 4 * kStripeCap;
    double *const sta = scut + kStripeCap, *const stb = sta + kStripeCap;
    double *const stc = stb + kStripeCap;
    unsigned long long *const slo = A.strlh + static_cast<size_t>(blockIdx.x) * 2 * kStripeCap;
    unsigned long long *const shi = slo + kStripeCap;
    const CellsDev &C = A.C;
    auto centre = [&](int j, bool v) {
        return v ? sx[j] + 0.5 * C.w[gid[j]] : sy[j] + 0.5 * C.h[gid[j]];
    };

    for (int task = blockIdx.x; task < A.ntasks; task += gridDim.x) {
        const SubTask T = A.tasks[task];
        const int size = T.e - T.b;
        if (tid == 0) {
            s_fail = size > kSub ? 1 : 0;
            s_nobst = 0;
            s_maxlen = 0;
            s_maxsteps = 0;
        }
        __syncthreads();
        if (s_fail) {
            if (tid == 0) A.fail[task] = 1;
            __syncthreads();
            continue;
        }
        for (int j = tid; j < size; j += nt) {
            const int32_t g = A.cells[T.b + j];
            gid[j] = g;
            sx[j] = C.x[g];
            sy[j] = C.y[g];
            sa[j] = C.area[g];
            at[j] = j;
        }
        for (int o = tid; o < A.F.K; o += nt) {
            const double *ob = A.F.obst + 4 * o;
            if (ob[2] <= T.box[0] || ob[0] >= T.box[2] || ob[3] <= T.box[1] || ob[1] >= T.box[3])
                continue;
            const int k = atomicAdd(&s_nobst, 1);
            if (k < kObstLocal)
                for (int q = 0; q < 4; ++q) obst[4 * k + q] = ob[q];
        }
        if (tid == 0) {
            SubDesc &d = cur0[0];
            for (int q = 0; q < 4; ++q) d.box[q] = T.box[q];
            d.b = 0;
            d.e = size;
            d.level = T.level;
            d.vert = T.vert;
            s_ncur = 1;
        }
        Free FL = A.F;
        {  // the rows overlapping the block, with their spans overlapping its x
           // range, into shared memory (the only spans its sub-boxes can meet)
            const int32_t r0 = first_row(A.F, T.box[1]);
            int32_t lo = r0, hi = A.F.R;  // first row from r0 with y start >= uy
            while (lo < hi) {
                const int32_t mid = (lo + hi) >> 1;
                if (A.F.rowy[2 * mid] < T.box[3]) lo = mid + 1;
                else hi = mid;
            }
            const int32_t nr = lo - r0;
            if (nr <= kRowsLocal) {
                for (int i = tid; i < nr; i += nt) {
                    const int64_t f = first_span(A.F, r0 + i, T.box[0]);
                    int64_t e = f;
                    while (e < A.F.rowspan[r0 + i + 1] && A.F.spans[2 * e] < T.box[2]) ++e;
                    scan[i] = static_cast<int32_t>(e - f);
                    lrowspan[i] = f;  // first span, global index (rebased below)
                }
                __syncthreads();
                const int32_t ns = cta_scan(scan, nr, warp_tmp);
                if (ns <= kSpansLocal) {
                    for (int i = tid; i < nr; i += nt) {
                        const int64_t f = lrowspan[i];
                        const int32_t o = scan[i];
                        const int32_t cnt = (i + 1 < nr ? scan[i + 1] : ns) - o;
                        for (int32_t q = 0; q < cnt; ++q) {
                            lspans[2 * (o + q)] = A.F.spans[2 * (f + q)];
                            lspans[2 * (o + q) + 1] = A.F.spans[2 * (f + q) + 1];
                        }
                        lrowy[2 * i] = A.F.rowy[2 * (r0 + i)];
                        lrowy[2 * i + 1] = A.F.rowy[2 * (r0 + i) + 1];
                    }
                    __syncthreads();
                    for (int i = tid; i <= nr; i += nt) lrowspan[i] = i < nr ? scan[i] : ns;
                    FL.rowy = lrowy;
                    FL.rowspan = lrowspan;
                    FL.spans = lspans;
                    FL.R = nr;
                }
            }
        }
        __syncthreads();
        if (s_nobst > kObstLocal && tid == 0) s_fail = 1;  // too many obstacles
        FL.obst = obst;
        FL.K = min(s_nobst, kObstLocal);
        SubDesc *cur = cur0, *nxt = cur0 + kMaxSub;
        for (;;) {
            __syncthreads();
            const int ncur = s_ncur;
            if (s_fail || ncur == 0) break;
            // A. which sub-blocks split at this level, their rank, the longest
            for (int i = tid; i < ncur; i += nt) {
                const int len = cur[i].e - cur[i].b;
                const int act = cur[i].level < A.max_level && len > A.min_cells;
                cur[i].act = act;
                scan[i] = act;
                if (act) atomicMax(&s_maxlen, len);
            }
            __syncthreads();
            const int nact = cta_scan(scan, ncur, warp_tmp);
            if (nact == 0) break;
            if (2 * nact > kMaxSub) {
                if (tid == 0) s_fail = 2;  // too many sub-blocks
                break;
            }
            const int maxlen = s_maxlen;
            for (int i = tid; i < ncur; i += nt) cur[i].rank = scan[i];
            __syncthreads();
            // the sub-blocks' starts, and ends with the split and axis flags,
            // in shared memory for the position lookups
            for (int i = tid; i < ncur; i += nt) {
                scan[i] = cur[i].b;
                scan[kMaxSub + i] = cur[i].e | (cur[i].act << 30) | (cur[i].vert << 29);
            }
            __syncthreads();
            // B. each position's sub-block; cells of each splitting sub-block by
            // (centre, id), ties by cell id as the reference's sortCells
            for (int p = tid; p < size; p += nt) {
                int lo = 0, hi = ncur;  // last sub-block with b <= p
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (scan[mid] <= p) lo = mid;
                    else hi = mid;
                }
                const int i = lo;
                const int ev = scan[kMaxSub + i];
                const bool in = p >= scan[i] && p < (ev & 0x1fffffff) && ((ev >> 30) & 1);
                dof[p] = static_cast<int16_t>(in ? i : -1);
                const int j = at[p];
                if (in) {
                    k2[p] = static_cast<uint32_t>(scan[i]);
                    k0[p] = ord(centre(j, ((ev >> 29) & 1) != 0));
                } else {
                    k2[p] = static_cast<uint32_t>(p);
                    k0[p] = 0ull;
                }
                k1[p] = (static_cast<unsigned long long>(gid[j]) << 32) | static_cast<unsigned>(j);
            }
            __syncthreads();
            {
                // the active sub-blocks in rank order: nxt is free until phase L
                for (int i = tid; i < ncur; i += nt)
                    if (cur[i].act) {
                        nxt[cur[i].rank].b = cur[i].b;
                        nxt[cur[i].rank].e = cur[i].e;
                    }
                __syncthreads();
                sort_segments(k0, k1, k2, nact, maxlen, [&](int g, int &b, int &e) {
                    b = nxt[g].b;
                    e = nxt[g].e;
                });
            }
            for (int p = tid; p < size; p += nt) at[p] = static_cast<int32_t>(k1[p] & 0xffffffffull);
            __syncthreads();
            if (A.exact) cta_prefix64(at, sa, size, A.scale, pre, w64);
            // C. areas and median in sorted order; the block profile's region
            {
                const Team tm(nact);
                for (int i = tm.team; i < ncur; i += tm.nteams) {
                    SubDesc &d = cur[i];
                    int32_t steps = 0, len = 0;
                    if (d.act) {
                        const bool v = d.vert != 0;
                        steps = v ? team_count_steps(tm, FL, d.box) : 0;
                        int32_t r0, r1;
                        box_rows(FL, d.box, r0, r1);
                        len = (v ? steps : 2 * (r1 - r0)) + 2;
                        if (tm.lane == 0) {
                            const int b = d.b, e = d.e, n = e - b;
                            double cell_area = 0.0, low = 0.0, high = 0.0;
                            int m = 0;
                            if (A.exact) {
                                m = median_fx(pre, b, n);
                                cell_area = static_cast<double>(pre[e] - pre[b]) * A.inv_scale;
                                low = static_cast<double>(pre[b + m] - pre[b]) * A.inv_scale;
                                high = static_cast<double>(pre[e] - pre[b + m]) * A.inv_scale;
                            } else {
                                for (int p = b; p < e; ++p) cell_area += sa[at[p]];
                                while (m + 1 < n && (m == 0 || low < 0.5 * cell_area))
                                    low += sa[at[b + m++]];
                                for (int p = b + m; p < e; ++p) high += sa[at[p]];
                            }
                            d.m = m;
                            d.cell_area = cell_area;
                            d.low_area = low;
                            d.high_area = high;
                            atomicMax(&s_maxsteps, steps);
                        }
                    }
                    if (tm.lane == 0) {
                        d.scnt = steps;
                        d.slen = len;
                        scan[i] = len;
                    }
                }
            }
            __syncthreads();
            const int tot = cta_scan(scan, ncur, warp_tmp);
            const int maxsteps = s_maxsteps;
            for (int i = tid; i < ncur; i += nt) cur[i].soff = scan[i];
            __syncthreads();  // every thread has read s_maxsteps before it is reset
            if (tid == 0) {
                s_maxsteps = 0;
                scan[ncur] = tot;
            }
            // D + E, in chunks of consecutive sub-blocks whose profile regions fit
            // the sort buffer together (scan[] holds the regions' offsets)
            for (int c0 = 0; c0 < ncur;) {
                if (tid == 0) {
                    int lo = c0 + 1, hi = ncur;  // the last end offset within reach
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (scan[mid] - scan[c0] <= kSortCap) lo = mid;
                        else hi = mid - 1;
                    }
                    int c1 = lo;
                    if (scan[c1] - scan[c0] > kSortCap) c1 = c0;  // one region too long
                    if (c1 == c0) s_fail = 3;  // sort buffer
                    s_c1 = c1;
                }
                __syncthreads();
                if (s_fail) break;
                const int c1 = s_c1, base = scan[c0];
                // D. the block profiles' regions: pads, then the steps sorted by (x, dh)
                {
                    const Team tm(nact);
                    for (int i = c0 + tm.team; i < c1; i += tm.nteams) {
                        const SubDesc &d = cur[i];
                        if (!d.act) continue;
                        const int o = d.soff - base;
                        team_emit_region(tm, FL, d.box, d.vert != 0, static_cast<uint32_t>(i), k0,
                                         k1, k2, o, d.slen);
                    }
                }
                __syncthreads();
                sort_segments(k0, k1, k2, c1 - c0, maxsteps, [&](int g, int &b, int &e) {
                        const SubDesc &d = cur[c0 + g];
                        const bool on = d.act && d.vert;
                        b = on ? d.soff - base + 2 : 0;
                        e = on ? d.soff - base + 2 + d.scnt : 0;
                    });
                // E. profile, cutline, half boxes, the halves' regions and stripe room
                {
                    const Team tm(nact);
                    for (int i = c0 + tm.team; i < c1; i += tm.nteams) {
                        SubDesc &d = cur[i];
                        if (!d.act) {
                            if (tm.lane == 0)
                                for (int side = 0; side < 2; ++side) d.hslen[side] = d.stcap[side] = 0;
                            continue;
                        }
                        const bool v = d.vert != 0;
                        const int o = d.soff - base;
                        const int64_t n = team_build_profile(tm, FL, d.box, v, k0, k1, o, d.scnt, d.slen);
                        const Prof room{reinterpret_cast<const double *>(k0 + o),
                                        reinterpret_cast<const double *>(k1 + o), n};
                        const double share = d.cell_area > 0.0 ? d.low_area / d.cell_area : 0.5;
                        const double lo = v ? d.box[0] : d.box[1], hi = v ? d.box[2] : d.box[3];
                        const double cut = room.total() > 0.0 ? room.coordinate_at(share * room.total())
                                                              : lo + share * (hi - lo);
                        double hb[8];
                        for (int q = 0; q < 4; ++q) hb[q] = hb[4 + q] = d.box[q];
                        hb[v ? 2 : 3] = cut;
                        hb[4 + (v ? 0 : 1)] = cut;
                        const double r_lo = room.before(cut);
                        int32_t hsc[2], hsl[2], cap[2];
                        for (int side = 0; side < 2; ++side) {
                            const double *bx = hb + 4 * side;
                            hsc[side] = v ? team_count_steps(tm, FL, bx) : 0;
                            int32_t r0, r1;
                            box_rows(FL, bx, r0, r1);
                            hsl[side] = (v ? hsc[side] : 2 * (r1 - r0)) + 2;
                            const int32_t k = team_count_obstacles(tm, FL, bx);
                            // stripes from midpoint splits hold more than half the split
                            // limit each: at most 2 room / limit of them (+ margin)
                            const double r_h = side ? ref_max(0.0, room.total() - r_lo) : r_lo;
                            const double lim = A.frac * (T.room > 0.0 ? T.room : r_h);
                            int32_t extra = A.stripe_extra;
                            if (T.room > 0.0 && lim > 0.0)
                                extra = static_cast<int32_t>(ref_min(static_cast<double>(A.stripe_extra),
                                                                     ceil(2.02 * r_h / lim) + 4.0));
                            cap[side] = 2 * k + 2 + extra;
                        }
                        tm.sync();  // every lane has read the profile and the box
                        if (tm.lane == 0) {
                            d.cut = cut;
                            for (int q = 0; q < 8; ++q) d.hbox[q] = hb[q];
                            for (int side = 0; side < 2; ++side) {
                                d.hscnt[side] = hsc[side];
                                d.hslen[side] = hsl[side];
                                d.stcap[side] = cap[side];
                                atomicMax(&s_maxsteps, hsc[side]);
                            }
                        }
                    }
                }
                __syncthreads();
                c0 = c1;
            }
            if (s_fail) break;
            // the halves' stripe offsets, then their profile regions' offsets
            for (int h = tid; h < 2 * ncur; h += nt) scan[h] = cur[h >> 1].stcap[h & 1];
            __syncthreads();
            const int stot = cta_scan(scan, 2 * ncur, warp_tmp);
            if (stot > kStripeCap) {
                if (tid == 0) s_fail = 4;  // stripes
                break;
            }
            for (int h = tid; h < 2 * ncur; h += nt) {
                cur[h >> 1].stoff[h & 1] = scan[h];
                scan[h] = cur[h >> 1].hslen[h & 1];
            }
            __syncthreads();
            const int htot = cta_scan(scan, 2 * ncur, warp_tmp);
            const int maxhsteps = s_maxsteps;
            for (int h = tid; h < 2 * ncur; h += nt) cur[h >> 1].hsoff[h & 1] = scan[h];
            __syncthreads();
            if (tid == 0) {
                s_maxsteps = 0;
                scan[2 * ncur] = htot;
            }
            // F + G, in chunks of consecutive halves
            for (int c0 = 0; c0 < 2 * ncur;) {
                if (tid == 0) {
                    const int nh = 2 * ncur;
                    int lo = c0 + 1, hi = nh;
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (scan[mid] - scan[c0] <= kSortCap) lo = mid;
                        else hi = mid - 1;
                    }
                    int c1 = lo;
                    if (scan[c1] - scan[c0] > kSortCap) c1 = c0;  // one region too long
                    if (c1 == c0) s_fail = 3;  // sort buffer
                    s_c1 = c1;
                }
                __syncthreads();
                if (s_fail) break;
                const int c1 = s_c1, base = scan[c0];
                // F. the halves' profile regions
                {
                    const Team tm(2 * nact);
                    for (int h = c0 + tm.team; h < c1; h += tm.nteams) {
                        const SubDesc &d = cur[h >> 1];
                        const int side = h & 1;
                        if (!d.act) continue;
                        const int o = d.hsoff[side] - base;
                        team_emit_region(tm, FL, d.hbox + 4 * side, d.vert != 0, static_cast<uint32_t>(h),
                                         k0, k1, k2, o, d.hslen[side]);
                    }
                }
                __syncthreads();
                sort_segments(k0, k1, k2, c1 - c0, maxhsteps, [&](int g, int &b, int &e) {
                        const int h = c0 + g;
                        const SubDesc &d = cur[h >> 1];
                        const bool on = d.act && d.vert;
                        b = on ? d.hsoff[h & 1] - base + 2 : 0;
                        e = on ? d.hsoff[h & 1] - base + 2 + d.hscnt[h & 1] : 0;
                    });
                // G. the halves' profiles and stripes
                {
                    const Team tm(2 * nact);
                    for (int h = c0 + tm.team; h < c1; h += tm.nteams) {
                        SubDesc &d = cur[h >> 1];
                        const int side = h & 1;
                        if (!d.act) continue;
                        const bool v = d.vert != 0;
                        const int o = d.hsoff[side] - base;
                        const int64_t n = team_build_profile(tm, FL, d.hbox + 4 * side, v, k0, k1, o,
                                                             d.hscnt[side], d.hslen[side]);
                        const int so = d.stoff[side];
                        int64_t ns = 0;
                        if (tm.lane == 0) {
                            const Prof room{reinterpret_cast<const double *>(k0 + o),
                                            reinterpret_cast<const double *>(k1 + o), n};
                            ns = make_stripes(room, d.hbox + 4 * side, v, side ? d.high_area : d.low_area,
                                              T.room, A.frac, A.limit_density, FL.obst, FL.K, d.cut,
                                              side == 0, scut + so, d.stcap[side], sta + so, stb + so,
                                              stc + so);
                            if (ns < 0) atomicExch(&s_fail, 4);
                            d.stcnt[side] = static_cast<int32_t>(ns < 0 ? 0 : ns);
                        }
                        ns = tm.bcast(ns);
                        for (int64_t q = tm.lane; q < ns; q += tm.T) {
                            slo[so + q] = ~0ull;
                            shi[so + q] = 0ull;
                        }
                    }
                }
                __syncthreads();
                if (s_fail) break;
                c0 = c1;
            }
            if (s_fail) break;
            // H. cells of each half by (-distance from the cut, id)
            for (int p = tid; p < size; p += nt) {
                const int i = dof[p];
                const int j = at[p];
                if (i >= 0) {
                    const SubDesc &d = cur[i];
                    const int mid = d.b + d.m;
                    const double c = centre(j, d.vert != 0);
                    const double from = p < mid ? d.cut - c : c - d.cut;
                    k2[p] = static_cast<uint32_t>(p < mid ? d.b : mid);
                    k0[p] = ord(-from);
                } else {
                    k2[p] = static_cast<uint32_t>(p);
                    k0[p] = 0ull;
                }
                k1[p] = (static_cast<unsigned long long>(gid[j]) << 32) | static_cast<unsigned>(j);
            }
            __syncthreads();
            {
                for (int i = tid; i < ncur; i += nt)
                    if (cur[i].act) {
                        nxt[cur[i].rank].b = cur[i].b;
                        nxt[cur[i].rank].e = cur[i].e;
                        nxt[cur[i].rank].m = cur[i].m;
                    }
                __syncthreads();
                sort_segments(k0, k1, k2, 2 * nact, maxlen, [&](int g, int &b, int &e) {
                    const SubDesc &d = nxt[g >> 1];
                    b = (g & 1) ? d.b + d.m : d.b;
                    e = (g & 1) ? d.e : d.b + d.m;
                });
            }
            for (int p = tid; p < size; p += nt) at[p] = static_cast<int32_t>(k1[p] & 0xffffffffull);
            __syncthreads();
            // I. greedy fill (exact areas: stripe starts by binary search on the
            // prefix, then each position looks its stripe up; else one thread
            // per half in the reference's order)
            if (A.exact) {
                cta_prefix64(at, sa, size, A.scale, pre, w64);
                for (int h = tid; h < 2 * ncur; h += nt) {
                    const SubDesc &d = cur[h >> 1];
                    if (!d.act) continue;
                    const int side = h & 1;
                    const int mid = d.b + d.m;
                    const int p0 = side ? mid : d.b, p1 = side ? d.e : mid;
                    const int ns = d.stcnt[side], so = d.stoff[side];
                    int q0 = p0;
                    for (int q = 0; q < ns; ++q) {
                        scut[so + q] = static_cast<double>(q0);  // stripe starts
                        if (q + 1 == ns) break;
                        const double cap = stc[so + q];
                        int lo = q0, hi = p1;
                        while (lo < hi) {
                            const int k = (lo + hi) >> 1;
                            if (static_cast<double>(pre[k] - pre[q0]) * A.inv_scale >= cap) hi = k;
                            else lo = k + 1;
                        }
                        q0 = lo;
                    }
                }
                __syncthreads();
                for (int p = tid; p < size; p += nt) {
                    const int i = dof[p];
                    if (i < 0) continue;
                    const SubDesc &d = cur[i];
                    const int side = p < d.b + d.m ? 0 : 1;
                    const int ns = d.stcnt[side], so = d.stoff[side];
                    int q = -1;
                    if (ns > 0) {
                        int lo = 0, hi = ns - 1;
                        while (lo < hi) {
                            const int k = (lo + hi + 1) >> 1;
                            if (scut[so + k] <= static_cast<double>(p)) lo = k;
                            else hi = k - 1;
                        }
                        q = so + lo;
                    }
                    sof[at[p]] = q;
                }
            } else {
                for (int h = tid; h < 2 * ncur; h += nt) {
                    const SubDesc &d = cur[h >> 1];
                    if (!d.act) continue;
                    const int side = h & 1;
                    const int mid = d.b + d.m;
                    const int p0 = side ? mid : d.b, p1 = side ? d.e : mid;
                    const int ns = d.stcnt[side], so = d.stoff[side];
                    if (ns == 0) {
                        for (int p = p0; p < p1; ++p) sof[at[p]] = -1;
                        continue;
                    }
                    int q = 0;
                    double used = 0.0;
                    for (int p = p0; p < p1; ++p) {
                        while (q + 1 < ns && used >= stc[so + q]) {
                            ++q;
                            used = 0.0;
                        }
                        const int j = at[p];
                        sof[j] = so + q;
                        used += sa[j];
                    }
                }
            }
            __syncthreads();
            // J. lowest and highest centre per stripe
            for (int p = tid; p < size; p += nt) {
                const int i = dof[p];
                if (i < 0) continue;
                const int j = at[p];
                const int q = sof[j];
                if (q < 0) continue;
                const unsigned long long o = ord(centre(j, cur[i].vert != 0));
                atomicMin(slo + q, o);
                atomicMax(shi + q, o);
            }
            __syncthreads();
            // K. new positions
            for (int p = tid; p < size; p += nt) {
                const int i = dof[p];
                if (i < 0) continue;
                const int j = at[p];
                const int q = sof[j];
                if (q < 0) continue;
                const bool v = cur[i].vert != 0;
                const double lo = unord(slo[q]), hi = unord(shi[q]);
                const double c0 = centre(j, v);
                const double t = hi > lo ? (c0 - lo) / (hi - lo) : 0.5;
                const double sz = v ? C.w[gid[j]] : C.h[gid[j]];
                const double a = sta[q], bb = stb[q];
                const double c = a + t * (bb - a);
                const double lim = ref_max(a, bb - sz);
                double np = c - 0.5 * sz;
                np = np < a ? a : (lim < np ? lim : np);
                (v ? sx : sy)[j] = np;
            }
            __syncthreads();
            // L. children: low and high halves, next axis
            for (int i = tid; i < ncur; i += nt) {
                const SubDesc &d = cur[i];
                if (!d.act) continue;
                for (int side = 0; side < 2; ++side) {
                    SubDesc &c = nxt[2 * d.rank + side];
                    for (int q = 0; q < 4; ++q) c.box[q] = d.hbox[4 * side + q];
                    c.b = side ? d.b + d.m : d.b;
                    c.e = side ? d.e : d.b + d.m;
                    c.level = d.level + 1;
                    c.vert = d.vert ? 0 : 1;
                }
            }
            if (tid == 0) {
                s_ncur = 2 * nact;
                s_maxlen = 0;
                s_maxsteps = 0;
            }
            SubDesc *t = cur;
            cur = nxt;
            nxt = t;
        }
        __syncthreads();
        if (s_fail) {
            if (tid == 0) A.fail[task] = s_fail;
        } else {
            for (int j = tid; j < size; j += nt) {
                C.x[gid[j]] = sx[j];
                C.y[gid[j]] = sy[j];
            }
            if (tid == 0) A.fail[task] = 0;
        }
        __syncthreads();
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
    DevBuf<long long> pre, tile;
    DevBuf<int32_t> sbeg;
    DevBuf<SubTask> tasks;
    DevBuf<int32_t> tfail;
    DevBuf<SubDesc> sdesc;
    DevBuf<double> sstrp;
    DevBuf<unsigned long long> sstrlh;
    bool subtree_attr = false;
    bool half_stripes_attr = false;
    // counters of the last ktg_lal call (ktg_lal_stats)
    double stats[16] = {};
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
    s->pre.release();
    s->tile.release();
    s->sbeg.release();
    s->tasks.release();
    s->tfail.release();
    s->sdesc.release();
    s->sstrp.release();
    s->sstrlh.release();
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

cudaError_t lal_sync(ktg_ctx *c) {
    c->lal->stats[3] += 1;
    return cudaStreamSynchronize(c->stream);
}

double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

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
    std::fill(s->stats, s->stats + 16, 0.0);
    const double t_start = now_ms();
    CellsDev C{x, y, c->width, c->height, c->area};
    const GridDev G{c->origin_x, c->origin_y, c->dx, c->dy, nx, ny};
    Free F{s->d_rowy.p, s->d_rowspan.p, s->d_spans.p, s->d_obst.p,
           static_cast<int32_t>(s->rowy.size() / 2), static_cast<int32_t>(s->obst.size() / 4)};
    const HostGrid HG{nx, ny, &c->avail_host, c->density_limit};
    std::vector<double> occ(nbins);
    auto refresh = [&]() -> int {  // bins and occupancy of the current positions
        const double t0 = now_ms();
        if (n > 0) {
            k_bins<<<blocks_for(n), kT, 0, c->stream>>>(C, n, G, s->binof.p);
            ++c->launches;
        }
        int r2 = launch_occupancy(c, x, y, s->occ.p, s->overflow.p);
        if (r2) return r2;
        KTG_CUDA(c, cudaMemcpyAsync(occ.data(), s->occ.p, sizeof(double) * nbins,
                                    cudaMemcpyDeviceToHost, c->stream));
        KTG_CUDA(c, lal_sync(c));
        s->stats[6] += now_ms() - t0;
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
    const int32_t stripe_extra =
        64 + static_cast<int32_t>(std::min(1048576.0, std::ceil(4.0 / frac)));
    const bool exact = c->area_shift >= 0 && c->lal_exact_sums != 0;
    const double scale = exact ? std::ldexp(1.0, c->area_shift) : 1.0;
    const double inv_scale = exact ? std::ldexp(1.0, -c->area_shift) : 1.0;

    // pre[p] = fixed-point area of cell positions [0, p), p <= count.
    auto fx_prefix = [&](int32_t count) -> int {
        const int32_t tiles = std::max(1, (count + kScanTile - 1) / kScanTile);
        int r2;
        if ((r2 = s->pre.ensure(c, static_cast<int64_t>(count) + 1)) ||
            (r2 = s->tile.ensure(c, tiles)))
            return r2;
        k_fx_tile_sums<<<tiles, kT, 0, c->stream>>>(s->cells.p, c->area, count, scale, s->tile.p);
        k_fx_tile_scan<<<1, kT, 0, c->stream>>>(s->tile.p, tiles);
        k_fx_prefix<<<tiles, kT, 0, c->stream>>>(s->cells.p, c->area, count, scale, s->tile.p,
                                                 s->pre.p);
        c->launches += 3;
        KTG_CUDA(c, cudaGetLastError());
        return KTG_OK;
    };

    // Blocks of at most kSub cells: one CTA each runs the rest of the
    // bisection; failed[t] = 1 for a block left for the level-by-level path.
    auto run_subtree = [&](const std::vector<SubTask> &tasks, std::vector<int32_t> &failed) -> int {
        const int32_t nt = static_cast<int32_t>(tasks.size());
        const int grid = std::max(1, std::min<int>(nt, c->num_sms));
        const double t0 = now_ms();
        int r2;
        if ((r2 = s->tasks.ensure(c, nt)) || (r2 = s->tfail.ensure(c, nt)) ||
            (r2 = s->sdesc.ensure(c, static_cast<int64_t>(grid) * 2 * kMaxSub)) ||
            (r2 = s->sstrp.ensure(c, static_cast<int64_t>(grid) * 4 * kStripeCap)) ||
            (r2 = s->sstrlh.ensure(c, static_cast<int64_t>(grid) * 2 * kStripeCap)))
            return r2;
        if (!s->subtree_attr) {
            KTG_CUDA(c, cudaFuncSetAttribute(k_subtree, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(kSubSmem)));
            s->subtree_attr = true;
        }
        KTG_CUDA(c, cudaMemcpyAsync(s->tasks.p, tasks.data(), sizeof(SubTask) * nt,
                                    cudaMemcpyHostToDevice, c->stream));
        SubArgs A{s->tasks.p, nt, s->tfail.p, s->cells.p, C, F, s->sdesc.p,
                  s->sstrp.p, s->sstrlh.p, max_level, min_cells, stripe_extra, frac,
                  c->density_limit, exact ? 1 : 0, scale, inv_scale};
        k_subtree<<<grid, kSubThreads, kSubSmem, c->stream>>>(A);
        ++c->launches;
        KTG_CUDA(c, cudaGetLastError());
        failed.assign(nt, 0);
        KTG_CUDA(c, cudaMemcpyAsync(failed.data(), s->tfail.p, sizeof(int32_t) * nt,
                                    cudaMemcpyDeviceToHost, c->stream));
        KTG_CUDA(c, lal_sync(c));
        s->stats[2] += 1;
        s->stats[4] += nt;
        s->stats[8] += now_ms() - t0;
        s->stats[10] += nt;
        for (int32_t t = 0; t < nt; ++t) {
            s->stats[11] += failed[t] != 0;
            if (failed[t] >= 1 && failed[t] <= 4) s->stats[11 + failed[t]] += 1;
        }
        return KTG_OK;
    };

    auto run_batch = [&]() -> int {
        const int32_t nreg = static_cast<int32_t>(batch.size());
        if (nreg == 0) return KTG_OK;
        const double t0 = now_ms();
        s->stats[0] += 1;
        s->stats[1] += nreg;
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
        KTG_CUDA(c, lal_sync(c));
        // level-1 blocks: one per region
        std::vector<int32_t> hb(nreg), he(nreg), hv(nreg, 1), hl(nreg, 1);
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
        for (;;) {
            // blocks that split: more than min_cells cells, below max_level;
            // small ones finish in the subtree kernel, the rest go level by level
            std::vector<int32_t> ab, ae, av, al;
            std::vector<double> abox, aroom;
            std::vector<SubTask> tasks;
            std::vector<size_t> task_src;
            auto take = [&](size_t k) {
                ab.push_back(hb[k]);
                ae.push_back(he[k]);
                av.push_back(hv[k]);
                al.push_back(hl[k]);
                for (int q = 0; q < 4; ++q) abox.push_back(hbox[4 * k + q]);
                aroom.push_back(hroom[k]);
            };
            for (size_t k = 0; k < hb.size(); ++k) {
                if (he[k] - hb[k] <= min_cells || hl[k] >= max_level) continue;
                if (he[k] - hb[k] <= c->lal_subtree_cells) {
                    SubTask t;
                    for (int q = 0; q < 4; ++q) t.box[q] = hbox[4 * k + q];
                    t.room = hroom[k];
                    t.b = hb[k];
                    t.e = he[k];
                    t.level = hl[k];
                    t.vert = hv[k];
                    tasks.push_back(t);
                    task_src.push_back(k);
                } else {
                    take(k);
                }
            }
            if (!tasks.empty()) {
                std::vector<int32_t> failed;
                if ((r2 = run_subtree(tasks, failed))) return r2;
                for (size_t t = 0; t < tasks.size(); ++t)
                    if (failed[t]) take(task_src[t]);
            }
            const int32_t na = static_cast<int32_t>(ab.size());
            if (na == 0) break;
            s->stats[2] += 1;
            s->stats[4] += na;
            s->stats[9] += 1;
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
            if ((r2 = seg_sort(c, s->keys.p, s->keys_tmp.p, segs, s->seg))) return r2;
            k_keys_to_cells<<<gcell, kT, 0, c->stream>>>(L, s->keys.p, s->cells.p);
            ++c->launches;
            // 2. areas, median, block profile bounds
            if (exact && (r2 = fx_prefix(run))) return r2;
            k_block_split<<<blocks_for(na), kT, 0, c->stream>>>(L, C, F, s->cells.p,
                                                              exact ? s->pre.p : nullptr, inv_scale);
            ++c->launches;
            std::vector<int64_t> bound(2 * na);
            KTG_CUDA(c, cudaMemcpyAsync(bound.data(), s->bound.p, sizeof(int64_t) * 2 * na,
                                        cudaMemcpyDeviceToHost, c->stream));
            KTG_CUDA(c, lal_sync(c));
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
            k_steps_cta<<<na, kT, 0, c->stream>>>(L, F, 0, s->soff.p, s->steps.p, s->nsteps.p);
            ++c->launches;
            std::vector<int64_t> nst(na);
            KTG_CUDA(c, cudaMemcpyAsync(nst.data(), s->nsteps.p, sizeof(int64_t) * na,
                                        cudaMemcpyDeviceToHost, c->stream));
            KTG_CUDA(c, lal_sync(c));
            std::vector<int64_t> ssegs;
            for (int32_t k = 0; k < na; ++k) {
                ssegs.push_back(soff[k]);
                ssegs.push_back(soff[k] + nst[k]);
            }
            if ((r2 = seg_sort(c, s->steps.p, s->steps_tmp.p, ssegs, s->seg))) return r2;
            // 3. profile, cutline, half boxes and bounds
            k_block_cut_cta<<<na, kT, 0, c->stream>>>(L, F, s->soff.p, s->steps.p, s->nsteps.p,
                                                      s->eoff.p, s->pe.p, s->pp.p, s->hbound.p);
            ++c->launches;
            std::vector<int64_t> hbound(4 * na);
            KTG_CUDA(c, cudaMemcpyAsync(hbound.data(), s->hbound.p, sizeof(int64_t) * 4 * na,
                                        cudaMemcpyDeviceToHost, c->stream));
            KTG_CUDA(c, lal_sync(c));
            std::vector<int64_t> hsoff(2 * na), heoff(2 * na), hcap(2 * na), stoff(2 * na);
            st = ed = 0;
            int64_t stripes = 0;
            for (int32_t h = 0; h < 2 * na; ++h) {
                hsoff[h] = st;
                st += hbound[2 * h];
                heoff[h] = ed;
                // pe: the profile edges; pp: the prefix, then up to `edges` cuts
                const int64_t edges = hbound[2 * h + 1] + stripe_extra;
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
            // cut capacity per half, read by k_half_stripes_cta
            KTG_CUDA(c, cudaMemcpyAsync(s->hbound.p, hcap.data(), sizeof(int64_t) * 2 * na, cudaMemcpyHostToDevice, c->stream));
            k_steps_cta<<<2 * na, kT, 0, c->stream>>>(L, F, 1, s->hsoff.p, s->steps.p, s->hnsteps.p);
            ++c->launches;
            std::vector<int64_t> hnst(2 * na);
            KTG_CUDA(c, cudaMemcpyAsync(hnst.data(), s->hnsteps.p, sizeof(int64_t) * 2 * na,
                                        cudaMemcpyDeviceToHost, c->stream));
            KTG_CUDA(c, lal_sync(c));
            ssegs.clear();
            for (int32_t h = 0; h < 2 * na; ++h) {
                ssegs.push_back(hsoff[h]);
                ssegs.push_back(hsoff[h] + hnst[h]);
            }
            if ((r2 = seg_sort(c, s->steps.p, s->steps_tmp.p, ssegs, s->seg))) return r2;
            // 4. stripes per half (profile arrays: e in pe, p and the cuts in pp)
            Stripes S{s->stoff.p, s->scount.p, s->sa.p, s->sb.p, s->scap.p, s->sused.p, s->slo.p, s->shi.p};
            if (!s->half_stripes_attr) {
                KTG_CUDA(c, cudaFuncSetAttribute(k_half_stripes_cta,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 static_cast<int>(kHalfStripesSmem)));
                s->half_stripes_attr = true;
            }
            k_half_stripes_cta<<<2 * na, kT, kHalfStripesSmem, c->stream>>>(
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
            KTG_CUDA(c, lal_sync(c));
            std::vector<int64_t> fsegs;
            for (int32_t k = 0; k < na; ++k) {
                fsegs.push_back(ab[k]);
                fsegs.push_back(ab[k] + mh[k]);
                fsegs.push_back(ab[k] + mh[k]);
                fsegs.push_back(ae[k]);
            }
            if ((r2 = seg_sort(c, s->keys.p, s->keys_tmp.p, fsegs, s->seg))) return r2;
            k_keys_to_cells<<<gcell, kT, 0, c->stream>>>(L, s->keys.p, s->cells.p);
            ++c->launches;
            if (exact) {
                if ((r2 = fx_prefix(run)) || (r2 = s->sbeg.ensure(c, stripes + 1))) return r2;
                k_fill_fx<<<2 * na, kT, 0, c->stream>>>(L, S, s->pre.p, inv_scale, s->sbeg.p);
                k_assign_fx<<<gcell, kT, 0, c->stream>>>(L, s->cells.p, S, s->sbeg.p,
                                                         s->stripe_of.p);
                c->launches += 2;
            } else {
                k_fill<<<blocks_for(2 * na), kT, 0, c->stream>>>(L, C, s->cells.p, S,
                                                                 s->stripe_of.p);
                ++c->launches;
            }
            k_stripe_minmax<<<gcell, kT, 0, c->stream>>>(L, C, s->cells.p, S, s->stripe_of.p);
            k_new_pos<<<gcell, kT, 0, c->stream>>>(L, C, s->cells.p, S, s->stripe_of.p);
            c->launches += 2;
            KTG_CUDA(c, cudaGetLastError());
            // children
            std::vector<double> halfbox(8 * na);
            KTG_CUDA(c, cudaMemcpyAsync(halfbox.data(), s->half_box.p, sizeof(double) * 8 * na,
                                        cudaMemcpyDeviceToHost, c->stream));
            KTG_CUDA(c, lal_sync(c));
            hb.clear();
            he.clear();
            hv.clear();
            hl.clear();
            hbox.clear();
            hroom.clear();
            for (int32_t k = 0; k < na; ++k) {
                for (int side = 0; side < 2; ++side) {
                    hb.push_back(side ? ab[k] + mh[k] : ab[k]);
                    he.push_back(side ? ae[k] : ab[k] + mh[k]);
                    hv.push_back(av[k] ? 0 : 1);
                    hl.push_back(al[k] + 1);
                    for (int q = 0; q < 4; ++q) hbox.push_back(halfbox[8 * k + 4 * side + q]);
                    hroom.push_back(aroom[k]);
                }
            }
        }
        batch.clear();
        batch_reach.clear();
        s->stats[5] += now_ms() - t0;
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
    s->stats[7] = now_ms() - t_start;
    return KTG_OK;
}

int lal_stats(ktg_ctx *c, double *out, int count) {
    for (int k = 0; k < count && k < 16; ++k) out[k] = c->lal ? c->lal->stats[k] : 0.0;
    return KTG_OK;
}

}  // namespace ktg
