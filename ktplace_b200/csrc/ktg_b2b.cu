// B2B net-model assembly and HPWL (sm_100a).
//
// Replaces LinearSystems::buildB2B / buildB2BAxis (globalPlacer/simpl/
// simpl_lss.cc:11-114) and simplPlacer::Impl::getHpwl (simpl_placer.cc:
// 256-275). Five launches build both axes at once:
//
//   k_bound_pins  one lane per net, pins staged by the warp: first-index
//                 argmin/argmax of the pin coordinate for x and y
//                 (simpl_lss.cc:32-45) and, from the same pass, the net's
//                 half perimeter (HPWL of the inputs).
//   k_row_count   one thread per (axis, movable cell): number of movable
//                 other ends of its B2B edges (simpl_lss.cc:75-83), plus a
//                 per-block total.
//   k_scan_blocks one block: exclusive scan of the block totals -> the first
//                 CSR slot of every block and nnz per axis.
//   k_fill        one thread per (axis, movable cell): block scan of the row
//                 counts -> row_ptr, then the row's edges in the reference's
//                 order (simpl_lss.cc:47-73, 89-113) so that diag and rhs are
//                 summed exactly as the reference sums them; rows with many
//                 movable other ends go to k_fill_heavy (a warp per row,
//                 the same edges, sums and roundings).
//
// Bit-exactness: the library is compiled with -fmad=false (no FMA
// contraction, like the reference's -ffp-contract=off) and CUDA's IEEE
// double division, so every w, val, diag and rhs equals the reference's.
//
// The same kernels also build Kraftwerk2's systems
// (Kraftwerk2Placer::Impl::buildSystem, globalPlacer/kraftwerk2/
// kraftwerk2_placer.cc:328-410) under its own rules (Rules = kKraftwerk2):
// the high bound pin is the last maximum (>=), the edge weight base is
// 2 w / (p - 1), nets may list a cell twice and edges to the row's own cell
// are skipped, the right-hand side uses the raw pin offsets, and there is
// neither an anchor term nor a diagonal floor (the caller applies them).
#include "ktg_common.cuh"
#include "ktg_context.h"

namespace ktg {
namespace {

constexpr int kBuildThreads = 256;
enum Rules { kSimpl = 0, kKraftwerk2 = 1 };

struct NetlistDev {
    const int32_t *var_of_vertex;
    const double *fixed_x;
    const double *fixed_y;
    const int32_t *net_start;
    const int32_t *pin_cell;
    const int32_t *pin_var;
    const double *off_x;
    const double *off_y;
    const double *net_base;
    const int32_t *net_mov;
    const int32_t *pin_start;
    const int2 *pin_ref;
    int32_t n;
    int32_t N;
};

NetlistDev view_of(const ktg_ctx *c) {
    return NetlistDev{c->var_of_vertex, c->fixed_x, c->fixed_y, c->net_start, c->pin_cell,
                      c->pin_var,       c->off_x,   c->off_y,   c->net_base,  c->net_mov,
                      c->pin_start,     c->pin_ref, static_cast<int32_t>(c->n),
                      static_cast<int32_t>(c->N)};
}

// Position of a pin's cell: movable cells read the variable vector, fixed
// cells their fixed coordinate (simpl_lss.cc:14-19).
__device__ __forceinline__ double cell_pos(const double *pos, const double *fixed, int32_t var,
                                           int32_t cell) {
    return var >= 0 ? pos[var] : fixed[cell];
}

// Pins staged per warp and round by k_bound_pins (two per lane).
constexpr int kPinChunk = 64;

// One lane per net, the pins staged by the warp. Each warp owns 32
// consecutive nets, whose pins are contiguous; the warp walks that pin range
// in chunks of kPinChunk, every lane loading and positioning pins of the
// chunk (coalesced pin reads, independent position gathers), and then each
// lane scans the part of its own net that falls in the chunk from shared
// memory, in pin order, carrying its running bounds across chunks. The scan
// order and the comparisons are the reference's, so the bound pins (first
// index wins on ties) and the half perimeters are the sequential ones; a
// net's term lands in the same thread as with one thread per net, so the
// block sums are too. WithBounds: also choose the bound pins of both axes.
template <bool WithBounds, int R = kSimpl>
__global__ void __launch_bounds__(kBuildThreads)
    k_bound_pins(NetlistDev nl, const double *__restrict__ x, const double *__restrict__ y,
                 uint32_t *__restrict__ lo_x, uint32_t *__restrict__ hi_x,
                 uint32_t *__restrict__ lo_y, uint32_t *__restrict__ hi_y,
                 double *__restrict__ partials, unsigned *__restrict__ ticket,
                 double *__restrict__ hpwl_out, double *__restrict__ terms = nullptr) {
    __shared__ double scratch[40];
    __shared__ double spx[kBuildThreads / 32][kPinChunk];
    __shared__ double spy[kBuildThreads / 32][kPinChunk];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int kw0 = blockIdx.x * blockDim.x + (wid << 5);  // the warp's first net
    int32_t s = 0, e = 0, p0 = 0, p1 = 0;
    if (k < nl.N) {
        s = nl.net_start[k];
        e = nl.net_start[k + 1];
    }
    if (kw0 < nl.N) {  // warp-uniform pin range of nets [kw0, kw0 + 32)
        p0 = nl.net_start[kw0];
        p1 = nl.net_start[min(kw0 + 32, nl.N)];
    }
    uint32_t lx = 0, hx = 0, ly = 0, hy = 0;
    double vlx = 0.0, vhx = 0.0, vly = 0.0, vhy = 0.0;
    // BBox::getEmpty then BBox::extend (geometry/kt_geometry.cc:70-75)
    double bx0 = __longlong_as_double(0x7ff0000000000000ll);  // +inf
    double by0 = bx0;
    double bx1 = -bx0;
    double by1 = -bx0;
    for (int32_t cb = p0; cb < p1; cb += kPinChunk) {
        for (int j = lane; j < kPinChunk; j += 32) {
            const int32_t p = cb + j;
            if (p < p1) {
                const int32_t cell = nl.pin_cell[p];
                const int32_t var = nl.pin_var[p];
                spx[wid][j] = cell_pos(x, nl.fixed_x, var, cell) + nl.off_x[p];
                spy[wid][j] = cell_pos(y, nl.fixed_y, var, cell) + nl.off_y[p];
            }
        }
        __syncwarp();
        const int32_t qa = max(s, cb), qb = min(e, cb + kPinChunk);
        for (int32_t p = qa; p < qb; ++p) {
            const int32_t q = p - s;
            const double px = spx[wid][p - cb];
            const double py = spy[wid][p - cb];
            if (WithBounds) {
                if (q == 0) {
                    vlx = vhx = px;
                    vly = vhy = py;
                } else {
                    // lo = pinAt(q) < pinAt(lo) ? q : lo (simpl_lss.cc:41-42);
                    // Kraftwerk2: hi = at[q] >= at[hi] ? q : hi (kraftwerk2_placer.cc:341-342)
                    if (px < vlx) { lx = q; vlx = px; }
                    if (R == kKraftwerk2 ? px >= vhx : px > vhx) { hx = q; vhx = px; }
                    if (py < vly) { ly = q; vly = py; }
                    if (R == kKraftwerk2 ? py >= vhy : py > vhy) { hy = q; vhy = py; }
                }
            }
            bx0 = ref_min(bx0, px);
            by0 = ref_min(by0, py);
            bx1 = ref_max(bx1, px);
            by1 = ref_max(by1, py);
        }
        __syncwarp();
    }
    double term = 0.0;
    if (k < nl.N) {
        if (WithBounds) {
            lo_x[k] = lx;
            hi_x[k] = hx;
            lo_y[k] = ly;
            hi_y[k] = hy;
        }
        // getHalfPerimeter: 0 for an empty box; nets with < 2 pins add 0.
        if (e - s >= 2 && !(bx0 > bx1 || by0 > by1)) term = (bx1 - bx0) + (by1 - by0);
        if (terms) terms[k] = term;
    }
    if (terms) return;  // summed in the reference's order by k_hpwl_ref_order
    const double bs = block_sum(term, scratch);
    if (threadIdx.x == 0) __stcg(partials + blockIdx.x, bs);
    if (last_block_done(ticket)) {
        const double total = sum_partials(partials, gridDim.x, scratch);
        if (threadIdx.x == 0) *hpwl_out = total;
    }
}

// HPWL in the reference's summation order (getDeterministicSum,
// simpl_parallel.h:35-51): the per-net terms in chunks of kGrain nets, each
// chunk summed left to right by one thread, then the chunk sums in order.
constexpr int64_t kGrain = 4096;
__global__ void __launch_bounds__(1024)
    k_hpwl_ref_order(const double *__restrict__ terms, int64_t N, double *__restrict__ out) {
    __shared__ double chunk[1024];
    const int64_t chunks = (N + kGrain - 1) / kGrain;
    double total = 0.0;
    for (int64_t c0 = 0; c0 < chunks; c0 += blockDim.x) {
        const int64_t c = c0 + threadIdx.x;
        double s = 0.0;
        if (c < chunks) {
            const int64_t e = min(N, (c + 1) * kGrain);
            for (int64_t i = c * kGrain; i < e; ++i) s += terms[i];
        }
        chunk[threadIdx.x] = s;
        __syncthreads();
        const int64_t here = chunks - c0 < blockDim.x ? chunks - c0 : blockDim.x;
        if (threadIdx.x == 0)
            for (int64_t k = 0; k < here; ++k) total += chunk[k];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = total;
}

// Edges of movable cell i's row on one axis, in the reference's order.
// Visit(cell_var, other_pos_of_cell, there, own_offset, w, raw own offset,
// raw other offset) for every edge.
template <int R = kSimpl, typename Visit>
__device__ __forceinline__ void for_each_edge(const NetlistDev &nl, const double *pos,
                                              const double *fixed, const double *off,
                                              const uint32_t *lo, const uint32_t *hi,
                                              double floor_len, int32_t i, Visit &&visit) {
    const double own_pos = pos[i];
    const int32_t e0 = nl.pin_start[i];
    const int32_t e1 = nl.pin_start[i + 1];
    for (int32_t e = e0; e < e1; ++e) {
        const int2 ref = nl.pin_ref[e];
        const int32_t k = ref.x;
        const uint32_t q = static_cast<uint32_t>(ref.y);
        const uint32_t l = lo[k];
        const uint32_t h = hi[k];
        if (l == h) continue;
        const int32_t s = nl.net_start[k];
        // Kraftwerk2's base, w * 2 / (p - 1), is exactly twice w / (p - 1)
        const double base = R == kKraftwerk2 ? 2.0 * nl.net_base[k] : nl.net_base[k];
        const double own_raw = off[s + q];
        const double own = own_pos + own_raw;
        const double own_offset = own - own_pos;
        auto edge = [&](uint32_t t) {
            const int32_t p = s + static_cast<int32_t>(t);
            const int32_t var = nl.pin_var[p];
            if (R == kKraftwerk2 && var == i) return;  // a second pin of the row's own cell
            const double cp = cell_pos(pos, fixed, var, nl.pin_cell[p]);
            const double there = cp + off[p];
            const double w = base / ref_max(fabs(own - there), floor_len);
            visit(var, cp, there, own_offset, w, own_raw, off[p]);
        };
        if (q == l || q == h) {
            const int32_t deg = nl.net_start[k + 1] - s;
            for (int32_t t = 0; t < deg; ++t)
                if (static_cast<uint32_t>(t) != q) edge(static_cast<uint32_t>(t));
        } else {
            edge(l);
            edge(h);
        }
    }
}

struct AxisArgs {
    const double *pos;
    const double *fixed;
    const double *off;
    const uint32_t *lo;
    const uint32_t *hi;
    double floor_len;
    const double *anchor;
    int32_t *row_ptr;
    int32_t *col;
    double *val;
    double *diag;
    double *rhs;
};

// Count of movable other ends per row; per-block totals for the scan.
template <int R = kSimpl>
__global__ void __launch_bounds__(kBuildThreads)
    k_row_count(NetlistDev nl, AxisArgs ax, AxisArgs ay, int32_t blocks_per_axis,
                int32_t *__restrict__ row_cnt, int64_t *__restrict__ block_sum_out) {
    __shared__ int32_t warp_tot[kBuildThreads / kWarp];
    const int axis = blockIdx.x >= blocks_per_axis ? 1 : 0;
    const AxisArgs &a = axis ? ay : ax;
    const int32_t i = (blockIdx.x - axis * blocks_per_axis) * blockDim.x + threadIdx.x;
    int32_t cnt = 0;
    if (i < nl.n) {
        const int32_t e0 = nl.pin_start[i];
        const int32_t e1 = nl.pin_start[i + 1];
        for (int32_t e = e0; e < e1; ++e) {
            const int2 ref = nl.pin_ref[e];
            const int32_t k = ref.x;
            const uint32_t q = static_cast<uint32_t>(ref.y);
            const uint32_t l = a.lo[k];
            const uint32_t h = a.hi[k];
            if (l == h) continue;
            const int32_t s = nl.net_start[k];
            if (R == kKraftwerk2) {
                // movable other ends that are not the row's own cell
                const auto other = [&](uint32_t t) {
                    const int32_t v = nl.pin_var[s + static_cast<int32_t>(t)];
                    return v >= 0 && v != i ? 1 : 0;
                };
                if (q == l || q == h) {
                    const int32_t deg = nl.net_start[k + 1] - s;
                    for (int32_t t = 0; t < deg; ++t)
                        if (static_cast<uint32_t>(t) != q) cnt += other(static_cast<uint32_t>(t));
                } else {
                    cnt += other(l) + other(h);
                }
            } else if (q == l || q == h) {
                cnt += nl.net_mov[k] - 1;  // every other movable pin of the net
            } else {
                cnt += (nl.pin_var[s + l] >= 0 ? 1 : 0) + (nl.pin_var[s + h] >= 0 ? 1 : 0);
            }
        }
        row_cnt[axis * nl.n + i] = cnt;
    }
    int32_t v = cnt;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) warp_tot[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int w = 0; w < kBuildThreads / kWarp; ++w) t += warp_tot[w];
        block_sum_out[blockIdx.x] = t;
    }
}

// Exclusive scan of the per-block totals of both axes (one block). Writes the
// first slot of every block in place, nnz per axis, row_ptr[n] and flags a
// capacity overflow.
__global__ void __launch_bounds__(1024)
    k_scan_blocks(int64_t *__restrict__ block_sum, int32_t blocks_per_axis, int32_t n,
                  int64_t cap, int32_t *__restrict__ row_ptr_x, int32_t *__restrict__ row_ptr_y,
                  int64_t *__restrict__ nnz_out, int *__restrict__ status) {
    __shared__ int64_t warp_tot[32];
    __shared__ int64_t carry;
    for (int axis = 0; axis < 2; ++axis) {
        int64_t *bs = block_sum + axis * blocks_per_axis;
        const int per = (blocks_per_axis + blockDim.x - 1) / blockDim.x;
        const int b0 = threadIdx.x * per;
        const int b1 = min(b0 + per, blocks_per_axis);
        int64_t local = 0;
        for (int b = b0; b < b1; ++b) local += bs[b];
        // block exclusive scan of `local`
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
            int64_t w = warp_tot[threadIdx.x];
            int64_t wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t t = __shfl_up_sync(0xffffffffu, wi, o);
                if (threadIdx.x >= o) wi += t;
            }
            warp_tot[threadIdx.x] = wi - w;  // exclusive warp offsets
            if (threadIdx.x == 31) carry = wi;
        }
        __syncthreads();
        int64_t run = warp_tot[threadIdx.x >> 5] + incl - local;
        for (int b = b0; b < b1; ++b) {
            const int64_t v = bs[b];
            bs[b] = run;
            run += v;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const int64_t total = carry;
            nnz_out[axis] = total;
            if (total > cap) {
                atomicCAS(status, kStatusOk, kStatusCapacity);
                (axis ? row_ptr_y : row_ptr_x)[n] = 0;
            } else {
                (axis ? row_ptr_y : row_ptr_x)[n] = static_cast<int32_t>(total);
            }
        }
        __syncthreads();
    }
}

// Row pointers from a block scan of the counts, then the row's entries.
// Kraftwerk2: alpha < 0 leaves the right-hand side at zero (withRhs false).
// Rows with at least this many movable other ends (the bound pins of large
// nets) are filled by k_fill_heavy, one warp per row, instead of by one
// thread: their edges are the long serial chains of dependent gathers that
// would otherwise set the kernel's time.
constexpr int32_t kHeavyRow = 32;

template <int R = kSimpl>
__global__ void __launch_bounds__(kBuildThreads, 4)
    k_fill(NetlistDev nl, AxisArgs ax, AxisArgs ay, int32_t blocks_per_axis, double alpha,
           const int32_t *__restrict__ row_cnt, const int64_t *__restrict__ block_first,
           int64_t cap, const int *__restrict__ status, int32_t *__restrict__ heavy) {
    __shared__ int32_t warp_tot[kBuildThreads / kWarp];
    const int axis = blockIdx.x >= blocks_per_axis ? 1 : 0;
    const AxisArgs &a = axis ? ay : ax;
    const int32_t i = (blockIdx.x - axis * blocks_per_axis) * blockDim.x + threadIdx.x;
    const int32_t cnt = (i < nl.n) ? row_cnt[axis * nl.n + i] : 0;
    // block exclusive scan of cnt
    int32_t incl = cnt;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[threadIdx.x >> 5] = incl;
    __syncthreads();
    if (threadIdx.x < 32) {
        const int32_t w = threadIdx.x < kBuildThreads / kWarp ? warp_tot[threadIdx.x] : 0;
        int32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (threadIdx.x >= o) wi += t;
        }
        if (threadIdx.x < kBuildThreads / kWarp) warp_tot[threadIdx.x] = wi - w;
    }
    __syncthreads();
    if (i >= nl.n) return;
    if (*status != kStatusOk) return;  // capacity exceeded: leave the buffers alone
    int64_t slot = block_first[blockIdx.x] + warp_tot[threadIdx.x >> 5] + (incl - cnt);
    a.row_ptr[i] = static_cast<int32_t>(slot);
    if (cnt >= kHeavyRow) {  // left for k_fill_heavy (the order of the list is free)
        heavy[1 + atomicAdd(heavy, 1)] = axis * nl.n + i;
        return;
    }
    double dg = 0.0;
    double rh = 0.0;
    for_each_edge<R>(nl, a.pos, a.fixed, a.off, a.lo, a.hi, a.floor_len, i,
                     [&](int32_t var, double cp, double there, double own_offset, double w,
                         double own_raw, double other_raw) {
                         dg += w;
                         if (var >= 0) {
                             if (slot < cap) {
                                 a.col[slot] = var;
                                 a.val[slot] = -w;
                             }
                             ++slot;
                             // Kraftwerk2: w * (otherOffset - ownOffset)
                             rh += R == kKraftwerk2 ? w * (other_raw - own_raw)
                                                    : w * ((there - cp) - own_offset);
                         } else {
                             // Kraftwerk2: w * (at[other] - ownOffset)
                             rh += R == kKraftwerk2 ? w * (there - own_raw)
                                                    : w * (there - own_offset);
                         }
                     });
    if (R == kKraftwerk2) {
        a.diag[i] = dg;
        a.rhs[i] = alpha < 0.0 ? 0.0 : rh;
        return;
    }
    if (alpha > 0.0) {
        const double p = a.pos[i];
        const double w = alpha / ref_max(fabs(p - a.anchor[i]), a.floor_len);
        dg += w;
        rh += w * a.anchor[i];
    }
    a.diag[i] = ref_max(dg, 1e-12);
    a.rhs[i] = rh;
}

// One warp per heavy row: the same edges in the same order as for_each_edge,
// 32 at a time. Each lane computes one edge (gathers, weight, the rhs term)
// and, when the other end is movable, writes its CSR entry at its rank among
// this chunk's entries; then every lane adds the chunk's w and rhs terms in
// edge order, so diag and rhs round exactly as in k_fill.
template <int R = kSimpl>
__global__ void __launch_bounds__(kBuildThreads)
    k_fill_heavy(NetlistDev nl, AxisArgs ax, AxisArgs ay, double alpha, int64_t cap,
                 const int *__restrict__ status, const int32_t *__restrict__ heavy) {
    const int lane = threadIdx.x & 31;
    const int32_t warps = static_cast<int32_t>((gridDim.x * blockDim.x) >> 5);
    const int32_t count = heavy[0];
    if (*status != kStatusOk) return;
    for (int32_t h = static_cast<int32_t>((blockIdx.x * blockDim.x + threadIdx.x) >> 5); h < count;
         h += warps) {
        const int32_t code = heavy[1 + h];
        const int axis = code >= nl.n ? 1 : 0;
        const int32_t i = code - (axis ? nl.n : 0);
        const AxisArgs &a = axis ? ay : ax;
        const double own_pos = a.pos[i];
        int64_t slot = a.row_ptr[i];
        double dg = 0.0, rh = 0.0;
        const int32_t e0 = nl.pin_start[i], e1 = nl.pin_start[i + 1];
        for (int32_t e = e0; e < e1; ++e) {
            const int2 ref = nl.pin_ref[e];
            const int32_t k = ref.x;
            const uint32_t q = static_cast<uint32_t>(ref.y);
            const uint32_t l = a.lo[k], hb = a.hi[k];
            if (l == hb) continue;
            const int32_t s0 = nl.net_start[k];
            const double base = R == kKraftwerk2 ? 2.0 * nl.net_base[k] : nl.net_base[k];
            const double own_raw = a.off[s0 + q];
            const double own = own_pos + own_raw;
            const double own_offset = own - own_pos;
            const bool bound = q == l || q == hb;
            // the pin's edges: every other pin t of the net, or its lo and hi
            const int32_t ne = bound ? nl.net_start[k + 1] - s0 : 2;
            for (int32_t t0 = 0; t0 < ne; t0 += 32) {
                const int32_t j = t0 + lane;
                bool has = false, entry = false;
                int32_t var = -1;
                double w = 0.0, term = 0.0;
                if (j < ne) {
                    const uint32_t t = bound ? static_cast<uint32_t>(j) : (j == 0 ? l : hb);
                    if (!bound || t != q) {
                        const int32_t p = s0 + static_cast<int32_t>(t);
                        var = nl.pin_var[p];
                        if (!(R == kKraftwerk2 && var == i)) {
                            has = true;
                            const double cp = cell_pos(a.pos, a.fixed, var, nl.pin_cell[p]);
                            const double other_raw = a.off[p];
                            const double there = cp + other_raw;
                            w = base / ref_max(fabs(own - there), a.floor_len);
                            if (var >= 0) {
                                entry = true;
                                term = R == kKraftwerk2 ? w * (other_raw - own_raw)
                                                        : w * ((there - cp) - own_offset);
                            } else {
                                term = R == kKraftwerk2 ? w * (there - own_raw)
                                                        : w * (there - own_offset);
                            }
                        }
                    }
                }
                const unsigned em = __ballot_sync(0xffffffffu, entry);
                if (entry) {
                    const int64_t at = slot + __popc(em & ((1u << lane) - 1u));
                    if (at < cap) {
                        a.col[at] = var;
                        a.val[at] = -w;
                    }
                }
                slot += __popc(em);
                const unsigned hm = __ballot_sync(0xffffffffu, has);
                for (unsigned m = hm; m; m &= m - 1) {  // edge order = lane order
                    const int src = __ffs(m) - 1;
                    dg += __shfl_sync(0xffffffffu, w, src);
                    rh += __shfl_sync(0xffffffffu, term, src);
                }
            }
        }
        if (lane == 0) {
            if (R == kKraftwerk2) {
                a.diag[i] = dg;
                a.rhs[i] = alpha < 0.0 ? 0.0 : rh;
            } else {
                if (alpha > 0.0) {
                    const double p = a.pos[i];
                    const double wa = alpha / ref_max(fabs(p - a.anchor[i]), a.floor_len);
                    dg += wa;
                    rh += wa * a.anchor[i];
                }
                a.diag[i] = ref_max(dg, 1e-12);
                a.rhs[i] = rh;
            }
        }
    }
}

// Kraftwerk2's adjustments after buildSystem: diag += move_weight and
// rhs = -move_weight * toward (kraftwerk2_placer.cc:716-721) when
// move_weight is given, then diag = max(diag, floor) when floor > 0
// (kraftwerk2_placer.cc:433-437).
__global__ void k_kw2_adjust(int32_t n, double *dx, double *rx, double *dy, double *ry,
                             const double *mw, const double *tx, const double *ty, double floor) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a = dx[i], b = dy[i];
    if (mw) {
        a += mw[i];
        b += mw[i];
        rx[i] = -mw[i] * tx[i];
        ry[i] = -mw[i] * ty[i];
    }
    if (floor > 0.0) {
        a = ref_max(a, floor);
        b = ref_max(b, floor);
    }
    dx[i] = a;
    dy[i] = b;
}


template <int R>
int launch_build(ktg_ctx *c, const double *x, const double *y, double alpha, const double *ax,
                 const double *ay, double floor_x, double floor_y) {
    const NetlistDev nl = view_of(c);
    const int32_t n = static_cast<int32_t>(c->n);
    const int net_blocks = static_cast<int>((c->N + kBuildThreads - 1) / kBuildThreads);
    const int32_t bpa = static_cast<int32_t>((c->n + kBuildThreads - 1) / kBuildThreads);
    KTG_CUDA(c, cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
    if (c->N > 0) {
        k_bound_pins<true, R><<<net_blocks, kBuildThreads, 0, c->stream>>>(
            nl, x, y, c->sys[0].lo, c->sys[0].hi, c->sys[1].lo, c->sys[1].hi, c->partials,
            c->counters + 0, c->scalars + 0);
        ++c->launches;
    } else {
        KTG_CUDA(c, cudaMemsetAsync(c->scalars + 0, 0, sizeof(double), c->stream));
    }
    AxisArgs a[2];
    for (int axis = 0; axis < 2; ++axis) {
        ktg::AxisSystem &s = c->sys[axis];
        a[axis] = AxisArgs{axis ? y : x, axis ? c->fixed_y : c->fixed_x, axis ? c->off_y : c->off_x,
                           s.lo, s.hi, axis ? floor_y : floor_x, axis ? ay : ax,
                           s.row_ptr, s.col, s.val, s.diag, s.rhs};
    }
    if (n > 0) {
        k_row_count<R><<<2 * bpa, kBuildThreads, 0, c->stream>>>(nl, a[0], a[1], bpa,
                                                                 c->row_cnt, c->block_sum);
        k_scan_blocks<<<1, 1024, 0, c->stream>>>(c->block_sum, bpa, n, c->cap_nnz,
                                                 c->sys[0].row_ptr, c->sys[1].row_ptr,
                                                 c->nnz_dev, c->status);
        KTG_CUDA(c, cudaMemsetAsync(c->heavy_rows, 0, sizeof(int32_t), c->stream));
        k_fill<R><<<2 * bpa, kBuildThreads, 0, c->stream>>>(nl, a[0], a[1], bpa, alpha,
                                                            c->row_cnt, c->block_sum, c->cap_nnz,
                                                            c->status, c->heavy_rows);
        k_fill_heavy<R><<<8 * c->num_sms, kBuildThreads, 0, c->stream>>>(
            nl, a[0], a[1], alpha, c->cap_nnz, c->status, c->heavy_rows);
        c->launches += 4;
    } else {
        KTG_CUDA(c, cudaMemsetAsync(c->sys[0].row_ptr, 0, sizeof(int32_t), c->stream));
        KTG_CUDA(c, cudaMemsetAsync(c->sys[1].row_ptr, 0, sizeof(int32_t), c->stream));
        KTG_CUDA(c, cudaMemsetAsync(c->nnz_dev, 0, 2 * sizeof(int64_t), c->stream));
    }
    KTG_CUDA(c, cudaGetLastError());
    return KTG_OK;
}

}  // namespace

int launch_build_b2b(ktg_ctx *c, const double *x, const double *y, double alpha,
                     const double *ax, const double *ay, double floor_x, double floor_y) {
    return launch_build<kSimpl>(c, x, y, alpha, ax, ay, floor_x, floor_y);
}

int launch_build_kraftwerk2(ktg_ctx *c, const double *x, const double *y, bool with_rhs,
                            double floor_x, double floor_y) {
    return launch_build<kKraftwerk2>(c, x, y, with_rhs ? 0.0 : -1.0, nullptr, nullptr, floor_x,
                                     floor_y);
}

int launch_kraftwerk2_adjust(ktg_ctx *c, const double *move_weight, const double *toward_x,
                             const double *toward_y, double diag_floor) {
    const int32_t n = static_cast<int32_t>(c->sys_n);
    if (n == 0) return KTG_OK;
    k_kw2_adjust<<<(n + 255) / 256, 256, 0, c->stream>>>(n, c->sys[0].diag, c->sys[0].rhs,
                                                        c->sys[1].diag, c->sys[1].rhs,
                                                        move_weight, toward_x, toward_y,
                                                        diag_floor);
    ++c->launches;
    KTG_CUDA(c, cudaGetLastError());
    return KTG_OK;
}

int launch_hpwl(ktg_ctx *c, const double *x, const double *y, double *out_dev) {
    if (c->N == 0) {
        KTG_CUDA(c, cudaMemsetAsync(out_dev, 0, sizeof(double), c->stream));
        return KTG_OK;
    }
    const NetlistDev nl = view_of(c);
    const int net_blocks = static_cast<int>((c->N + kBuildThreads - 1) / kBuildThreads);
    if (c->hpwl_order == 2) {
        if (c->hpwl_terms_cap < c->N) {
            if (c->hpwl_terms) cudaFree(c->hpwl_terms);
            c->hpwl_terms = nullptr;
            KTG_CUDA(c, cudaMalloc(&c->hpwl_terms, sizeof(double) * c->N));
            c->hpwl_terms_cap = c->N;
        }
        k_bound_pins<false><<<net_blocks, kBuildThreads, 0, c->stream>>>(
            nl, x, y, nullptr, nullptr, nullptr, nullptr, c->partials, c->counters + 0, out_dev,
            c->hpwl_terms);
        k_hpwl_ref_order<<<1, 1024, 0, c->stream>>>(c->hpwl_terms, c->N, out_dev);
        c->launches += 2;
        KTG_CUDA(c, cudaGetLastError());
        return KTG_OK;
    }
    k_bound_pins<false><<<net_blocks, kBuildThreads, 0, c->stream>>>(
        nl, x, y, nullptr, nullptr, nullptr, nullptr, c->partials, c->counters + 0, out_dev);
    ++c->launches;
    KTG_CUDA(c, cudaGetLastError());
    return KTG_OK;
}

}  // namespace ktg
