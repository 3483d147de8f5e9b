/* Plain-C restatement of KTPlace's SimPL quadratic-solve path.
 *
 * TEST INFRASTRUCTURE ONLY (see ktp_oracle.h). Each function names the
 * reference lines it restates. Single-threaded; the reference's TBB
 * parallelism only changes which thread computes a row, never a result
 * (per-row outputs are independent and reductions use fixed 4096 chunks).
 */
#include "ktp_oracle.h"

#include <math.h>
#include <stddef.h>
#include <stdlib.h>

#define KTO_GRAIN 4096

/* std::max / std::min / std::clamp as the reference uses them:
 * max(a, b) = (a < b) ? b : a, min(a, b) = (b < a) ? b : a. */
static inline double kmax(double a, double b) { return (a < b) ? b : a; }
static inline double kmin(double a, double b) { return (b < a) ? b : a; }

/* simpl_parallel.h:35-51 */
double kto_dot(int64_t n, const double *a, const double *b) {
    const int64_t chunks = (n + KTO_GRAIN - 1) / KTO_GRAIN;
    double total = 0.0;
    for (int64_t c = 0; c < chunks; ++c) {
        const int64_t end = (c + 1) * KTO_GRAIN < n ? (c + 1) * KTO_GRAIN : n;
        double sum = 0.0;
        for (int64_t i = c * KTO_GRAIN; i < end; ++i) sum += a[i] * b[i];
        total += sum;
    }
    return total;
}

/* Position of vertex v on the axis: movable vertices read pos_mov through
 * their variable, fixed ones the fixed coordinate (simpl_lss.cc:14-19). */
static inline double vpos(const kto_netlist *nl, int vertical, const double *pos_mov, int32_t v) {
    const int32_t var = nl->var_of_vertex[v];
    if (var >= 0) return pos_mov[var];
    return vertical ? nl->fixed_x[v] : nl->fixed_y[v];
}

static inline double pin_at(const kto_netlist *nl, int vertical, const double *pos_mov,
                            int64_t p) {
    return vpos(nl, vertical, pos_mov, nl->pin_cell[p]) + (vertical ? nl->off_x[p] : nl->off_y[p]);
}

/* simpl_lss.cc:29-114 */
int kto_b2b_axis(const kto_netlist *nl, int vertical, const double *pos_mov, double floor_len,
                 double alpha, const double *anchor, uint32_t *lo, uint32_t *hi,
                 int64_t *row_ptr, int32_t *col, double *val, int64_t cap, double *diag,
                 double *rhs) {
    const int64_t N = nl->num_nets;
    const int64_t n = nl->num_movable;
    /* Bound pins, first index wins ties (simpl_lss.cc:32-45). */
    for (int64_t k = 0; k < N; ++k) {
        const int64_t s = nl->net_start[k];
        const int64_t deg = nl->net_start[k + 1] - s;
        uint32_t l = 0, h = 0;
        for (uint32_t q = 1; q < deg; ++q) {
            const double v = pin_at(nl, vertical, pos_mov, s + q);
            l = v < pin_at(nl, vertical, pos_mov, s + l) ? q : l;
            h = v > pin_at(nl, vertical, pos_mov, s + h) ? q : h;
        }
        lo[k] = l;
        hi[k] = h;
    }
    /* Count pass (simpl_lss.cc:75-83) then the fill pass (:89-113); both walk
     * forEachEdge (:47-73). */
    row_ptr[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        const int pass_fill = col != NULL;
        int64_t count = 0;
        int64_t slot = pass_fill ? row_ptr[i] : 0;
        double dg = 0.0, rh = 0.0;
        for (int64_t e = nl->pin_start[i]; e < nl->pin_start[i + 1]; ++e) {
            const int32_t k = nl->pin_net[e];
            const uint32_t q = (uint32_t)nl->pin_q[e];
            const uint32_t l = lo[k], h = hi[k];
            if (l == h) continue;
            const int64_t s = nl->net_start[k];
            const int64_t deg = nl->net_start[k + 1] - s;
            const double base = nl->net_weight[k] / (double)(deg - 1);
            const double own = pin_at(nl, vertical, pos_mov, s + q);
            const double own_pos = vpos(nl, vertical, pos_mov, nl->pin_cell[s + q]);
            const double own_offset = own - own_pos;
            uint32_t list2[2] = {l, h};
            const int bound = (q == l || q == h);
            const uint32_t m = bound ? (uint32_t)deg : 2u;
            for (uint32_t t = 0; t < m; ++t) {
                const uint32_t other = bound ? t : list2[t];
                if (bound && other == q) continue;
                const int32_t cell = nl->pin_cell[s + other];
                const double there = pin_at(nl, vertical, pos_mov, s + other);
                const double w = base / kmax(fabs(own - there), floor_len);
                const int32_t var = nl->var_of_vertex[cell];
                if (!pass_fill) {
                    count += var >= 0 ? 1 : 0;
                    continue;
                }
                dg += w;
                if (var >= 0) {
                    if (slot >= cap) return -1;
                    col[slot] = var;
                    val[slot] = -w;
                    ++slot;
                    rh += w * ((there - vpos(nl, vertical, pos_mov, cell)) - own_offset);
                } else {
                    rh += w * (there - own_offset);
                }
            }
        }
        if (!pass_fill) {
            row_ptr[i + 1] = row_ptr[i] + count;
            continue;
        }
        if (alpha > 0.0) {
            const double p = pos_mov[i];
            const double w = alpha / kmax(fabs(p - anchor[i]), floor_len);
            dg += w;
            rh += w * anchor[i];
        }
        diag[i] = kmax(dg, 1e-12);
        rhs[i] = rh;
    }
    return 0;
}

/* SparseSystem::multiply (simpl_lss.h:49-57) */
static void spmv(int64_t n, const int64_t *row_ptr, const int32_t *col, const double *val,
                 const double *diag, const double *in, double *out) {
    for (int64_t i = 0; i < n; ++i) {
        double sum = diag[i] * in[i];
        for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) sum += val[e] * in[col[e]];
        out[i] = sum;
    }
}

/* simpl_lss.cc:203-290, one axis (the two axes of the reference loop never
 * interact: each steps while it is live, with the shared iteration cap). */
int kto_pcg_axis(int64_t n, const int64_t *row_ptr, const int32_t *col, const double *val,
                 const double *diag, const double *rhs, double *x, double tol, int64_t max_iter,
                 double *resid_out, int64_t *iters, double *hist, int64_t hist_cap) {
    double *r = calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    double *z = calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    double *p = calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    double *ap = calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    if (!r || !z || !p || !ap) {
        free(r), free(z), free(p), free(ap);
        return -1;
    }
    double resid = 0.0, rho = 0.0;
    int active = 0;
    spmv(n, row_ptr, col, val, diag, x, ap);
    for (int64_t i = 0; i < n; ++i) {
        r[i] = rhs[i] - ap[i];
        z[i] = r[i] / diag[i];
    }
    const double b_norm = sqrt(kto_dot(n, rhs, rhs));
    if (b_norm > 0.0) {
        for (int64_t i = 0; i < n; ++i) p[i] = z[i];
        rho = kto_dot(n, r, z);
        resid = sqrt(kto_dot(n, r, r)) / b_norm;
        active = 1;
    }
    int64_t it = 0;
    while (it < max_iter && active && resid > tol) {
        spmv(n, row_ptr, col, val, diag, p, ap);
        const double pap = kto_dot(n, p, ap);
        int ok = pap > 0.0;
        if (ok) {
            const double a = rho / pap;
            for (int64_t i = 0; i < n; ++i) {
                x[i] += a * p[i];
                r[i] -= a * ap[i];
                z[i] = r[i] / diag[i];
            }
            resid = sqrt(kto_dot(n, r, r)) / b_norm;
            const double rho_next = kto_dot(n, r, z);
            ok = rho_next > 0.0;
            if (ok) {
                const double beta = rho_next / rho;
                for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
                rho = rho_next;
            }
        }
        if (!ok) active = 0;
        if (hist != NULL && it < hist_cap) hist[it] = resid;
        ++it;
    }
    *resid_out = resid;
    *iters = it;
    free(r), free(z), free(p), free(ap);
    return 0;
}

/* One net's half perimeter (simpl_placer.cc:265-273, BBox::extend and
 * getHalfPerimeter in geometry/kt_geometry.cc:35-75). */
static double net_hpwl(const kto_netlist *nl, const double *x, const double *y, int64_t k) {
    const int64_t s = nl->net_start[k];
    const int64_t e = nl->net_start[k + 1];
    if (e - s < 2) return 0.0;
    double lx = INFINITY, ly = INFINITY, ux = -INFINITY, uy = -INFINITY;
    for (int64_t p = s; p < e; ++p) {
        const double px = vpos(nl, 1, x, nl->pin_cell[p]) + nl->off_x[p];
        const double py = vpos(nl, 0, y, nl->pin_cell[p]) + nl->off_y[p];
        lx = kmin(lx, px);
        ly = kmin(ly, py);
        ux = kmax(ux, px);
        uy = kmax(uy, py);
    }
    if (lx > ux || ly > uy) return 0.0;
    return (ux - lx) + (uy - ly);
}

void kto_hpwl_terms(const kto_netlist *nl, const double *x, const double *y, double *out) {
    for (int64_t k = 0; k < nl->num_nets; ++k) out[k] = net_hpwl(nl, x, y, k);
}

/* simpl_placer.cc:256-275 with getDeterministicSum (simpl_parallel.h:35-51) */
double kto_hpwl(const kto_netlist *nl, const double *x, const double *y) {
    const int64_t N = nl->num_nets;
    const int64_t chunks = (N + KTO_GRAIN - 1) / KTO_GRAIN;
    double total = 0.0;
    for (int64_t c = 0; c < chunks; ++c) {
        const int64_t end = (c + 1) * KTO_GRAIN < N ? (c + 1) * KTO_GRAIN : N;
        double sum = 0.0;
        for (int64_t k = c * KTO_GRAIN; k < end; ++k) sum += net_hpwl(nl, x, y, k);
        total += sum;
    }
    return total;
}

/* BinGrid::clampIndex (simpl_grid.h:125-127) */
static inline int64_t clamp_index(double f, int64_t n) {
    const double hi = (double)n - 1e-9;
    const double c = f < 0.0 ? 0.0 : (hi < f ? hi : f);
    return (int64_t)c;
}

/* simpl_placer.cc:277-289 and BinGrid::getBinOf (simpl_grid.h:82-90) */
void kto_occupancy(int64_t n, const double *x, const double *y, const double *width,
                   const double *height, const double *area, double origin_x, double origin_y,
                   double dx, double dy, int64_t nx, int64_t ny, double *occ) {
    for (int64_t k = 0; k < nx * ny; ++k) occ[k] = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double cx = x[i] + 0.5 * width[i];
        const double cy = y[i] + 0.5 * height[i];
        const int64_t ix = clamp_index((cx - origin_x) / dx, nx);
        const int64_t iy = clamp_index((cy - origin_y) / dy, ny);
        occ[iy * nx + ix] += area[i];
    }
}

/* simpl_placer.cc:291-297 */
double kto_overflow(int64_t bins, const double *occ, const double *avail, double density_limit,
                    double total_avail) {
    double excess = 0.0;
    for (int64_t k = 0; k < bins; ++k) excess += kmax(occ[k] - density_limit * avail[k], 0.0);
    return total_avail > 0.0 ? excess / total_avail : 0.0;
}
