/* Plain-C restatement of KTPlace's SimPL quadratic-solve path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker that the CUDA path is compared with.
 * It is pinned against the reference's own code (oracle/_ref, built from the
 * reference sources) and against the golden vectors under tests/golden/.
 * Nothing in the product links or calls it.
 *
 * Compiled with -ffp-contract=off, as the reference is (src/Master.make:21),
 * so every expression rounds exactly as the reference's does.
 */
#ifndef KTP_ORACLE_H
#define KTP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* SimPL's flattened netlist (globalPlacer/simpl/simpl_lss.h:27-36) as SoA. */
typedef struct {
    int64_t num_vertices;
    int64_t num_movable;
    int64_t num_nets;
    const int32_t *mov_vertex;    /* [n] */
    const int32_t *var_of_vertex; /* [V], -1 = fixed */
    const double *fixed_x;        /* [V] */
    const double *fixed_y;        /* [V] */
    const int64_t *net_start;     /* [N+1] */
    const int32_t *pin_cell;      /* [P] */
    const double *off_x;          /* [P] */
    const double *off_y;          /* [P] */
    const double *net_weight;     /* [N] */
    const int64_t *pin_start;     /* [n+1] */
    const int32_t *pin_net;       /* [Pm] */
    const int32_t *pin_q;         /* [Pm] */
} kto_netlist;

/* One axis of LinearSystems::buildB2B (simpl_lss.cc:11-114).
 * pos_mov: movable positions along the axis (x for vertical != 0).
 * anchor may be NULL when alpha <= 0.
 * Outputs: lo/hi [N] bound pin indices; row_ptr [n+1]. When col is NULL only
 * the bound pins and row_ptr are produced (count pass); otherwise col/val
 * (capacity cap), diag [n] and rhs [n] are filled.
 * Returns 0, or -1 when cap is too small. */
int kto_b2b_axis(const kto_netlist *nl, int vertical, const double *pos_mov, double floor_len,
                 double alpha, const double *anchor, uint32_t *lo, uint32_t *hi,
                 int64_t *row_ptr, int32_t *col, double *val, int64_t cap, double *diag,
                 double *rhs);

/* One axis of solveBothAxes (simpl_lss.cc:203-290): Jacobi-PCG, warm start x,
 * stop when the recursive relative residual <= tol or after max_iter steps,
 * stop early on non-positive p.Ap or r.z. hist (may be NULL) receives the
 * residual after each step (capacity hist_cap).
 * Outputs: *resid (final relative residual, 0 when ||b|| == 0), *iters. */
int kto_pcg_axis(int64_t n, const int64_t *row_ptr, const int32_t *col, const double *val,
                 const double *diag, const double *rhs, double *x, double tol, int64_t max_iter,
                 double *resid, int64_t *iters, double *hist, int64_t hist_cap);

/* simplPlacer::Impl::getHpwl (simpl_placer.cc:256-275). */
double kto_hpwl(const kto_netlist *nl, const double *x, const double *y);

/* Per-net half perimeters (the terms of kto_hpwl). */
void kto_hpwl_terms(const kto_netlist *nl, const double *x, const double *y, double *out);

/* Impl::getOccupancy (simpl_placer.cc:282-289) on a nx x ny grid. */
void kto_occupancy(int64_t n, const double *x, const double *y, const double *width,
                   const double *height, const double *area, double origin_x, double origin_y,
                   double dx, double dy, int64_t nx, int64_t ny, double *occ);

/* Impl::getOverflow (simpl_placer.cc:291-297). */
double kto_overflow(int64_t bins, const double *occ, const double *avail, double density_limit,
                    double total_avail);

/* getDeterministicSum / getDot (simpl_parallel.h:35-57): 4096-element chunks
 * summed in order, partials summed in order. */
double kto_dot(int64_t n, const double *a, const double *b);

#ifdef __cplusplus
}
#endif

#endif
