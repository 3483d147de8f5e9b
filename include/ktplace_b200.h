/* ktplace_b200 — B200 (sm_100a) implementation of KTPlace's SimPL
 * quadratic-solve hot path, exposed as a C ABI.
 *
 * The path has three parts, each replacing a reference function:
 *   - B2B net-model assembly into CSR for x and y
 *       LinearSystems::buildB2B   globalPlacer/simpl/simpl_lss.cc:11-114
 *   - Jacobi-preconditioned CG on both systems
 *       solveBothAxes             globalPlacer/simpl/simpl_lss.cc:203-290
 *       (SparseSystem::multiply   globalPlacer/simpl/simpl_lss.h:49-57)
 *   - HPWL and density-bin reductions
 *       simplPlacer::Impl::getHpwl / getOccupancy / getOverflow
 *                                 globalPlacer/simpl/simpl_placer.cc:256-297
 *
 * Conventions
 *   - Every entry point returns KTG_OK (0) or a negative KTG_ERR_* code and
 *     never throws; ktg_last_error() describes the last failure.
 *   - One context owns one device, one CUDA stream and the device-resident
 *     netlist and systems. A context is not thread-safe; use one per thread.
 *   - Pointer mode (ktg_set_pointer_mode) decides how vector and scalar
 *     arguments are read:
 *       KTG_PTR_HOST   (default) host memory; the call copies in and out and
 *                      returns after the results are in host memory.
 *       KTG_PTR_DEVICE device memory of the context's device; the call only
 *                      enqueues work on the context's stream (scalar outputs
 *                      are written to device memory too).
 *     Netlist, grid and system upload/download arguments are always host
 *     memory.
 *   - Indices are 0-based. Movable cell i is variable i; vertices include the
 *     fixed cells. A netlist's pins must be deduplicated per cell and sorted
 *     by cell id inside each net, as SimPL's collectNets does
 *     (globalPlacer/simpl/simpl_dm.cc:49-63).
 */
#ifndef KTPLACE_B200_H
#define KTPLACE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KTG_OK 0
#define KTG_ERR_ARG (-1)      /* bad argument or size                       */
#define KTG_ERR_CUDA (-2)     /* a CUDA runtime call failed                 */
#define KTG_ERR_NOMEM (-3)    /* device or host allocation failed           */
#define KTG_ERR_STATE (-4)    /* call out of order (e.g. no netlist yet)    */
#define KTG_ERR_TIMEOUT (-5)  /* a bounded device wait gave up              */
#define KTG_ERR_RANGE (-6)    /* a size exceeds the 32-bit index range      */

#define KTG_PTR_HOST 0
#define KTG_PTR_DEVICE 1

#define KTG_AXIS_X 0
#define KTG_AXIS_Y 1

typedef struct ktg_ctx ktg_ctx;

/* SimPL's flattened netlist (Netlist, globalPlacer/simpl/simpl_lss.h:27-36)
 * as structure-of-arrays. All pointers are host memory. */
typedef struct {
    int64_t num_vertices;          /* V: movable + fixed                       */
    int64_t num_movable;           /* n                                        */
    int64_t num_nets;              /* N                                        */
    const int32_t *mov_vertex;     /* [n]   vertex of variable i (movVertex)   */
    const int32_t *var_of_vertex;  /* [V]   variable of vertex, -1 when fixed  */
    const double *fixed_x;         /* [V]   vertex positions (fixedX)          */
    const double *fixed_y;         /* [V]                                      */
    const int64_t *net_start;      /* [N+1] pins of net k: [net_start[k], ..)  */
    const int32_t *pin_cell;       /* [P]   vertex of each pin (NetPins.cells) */
    const double *off_x;           /* [P]   lower-left-relative pin offsets    */
    const double *off_y;           /* [P]                                      */
    const double *net_weight;      /* [N]                                      */
    const int64_t *pin_start;      /* [n+1] cell -> (net, pin) CSR (pinStart)  */
    const int32_t *pin_net;        /* [Pm]  pinsOfCell[e].net                  */
    const int32_t *pin_q;          /* [Pm]  pinsOfCell[e].pin                  */
    const double *width;           /* [n]   movable cell widths (density)      */
    const double *height;          /* [n]   movable cell heights               */
} ktg_netlist_view;

/* SimPL's bin grid (BinGrid, globalPlacer/simpl/simpl_grid.h:67-128). Bin
 * (ix, iy) is element iy * nx + ix. Host memory. */
typedef struct {
    double origin_x;
    double origin_y;
    double dx;
    double dy;
    int64_t nx;
    int64_t ny;
    const double *avail;           /* [nx*ny] free row area per bin            */
    double total_avail;
    double density_limit;          /* g of getOverflow, clamped to [0.05, 1]   */
} ktg_grid_view;

/* Result of one ktg_solve: the last relative residual of each axis (the
 * Residuals of solveBothAxes) and the number of lock-step iterations. */
typedef struct {
    double resid_x;
    double resid_y;
    int64_t iters;                 /* loop iterations, as the observer counts  */
    int64_t iters_x;               /* steps taken by the x axis                */
    int64_t iters_y;
    int32_t status;                /* KTG_OK or KTG_ERR_TIMEOUT                */
    int32_t live;                  /* bit 0 / bit 1: x / y still live at exit  */
} ktg_solve_info;

/* ---- context ------------------------------------------------------------ */

/* Creates a context on CUDA device `device`. No reference counterpart: the
 * reference owns its systems as members of simplPlacer::Impl
 * (simpl_placer.cc:158-159). */
int ktg_create(int device, ktg_ctx **out);
void ktg_destroy(ktg_ctx *ctx);
const char *ktg_last_error(const ktg_ctx *ctx);
const char *ktg_version(void);

/* Work is enqueued on `stream` (a cudaStream_t); NULL selects the context's
 * own stream. */
int ktg_set_stream(ktg_ctx *ctx, void *stream);
int ktg_set_pointer_mode(ktg_ctx *ctx, int mode);

/* ---- netlist ------------------------------------------------------------ */

/* Uploads the netlist topology once per design; it stays device-resident.
 * Replaces the per-call reads of Netlist in buildB2B and getHpwl
 * (simpl_lss.cc:11-27, simpl_placer.cc:256-275). */
int ktg_upload_netlist(ktg_ctx *ctx, const ktg_netlist_view *nl);

/* ---- B2B assembly --------------------------------------------------------- */

/* LinearSystems::buildB2B (simpl_lss.cc:11-114) for both axes. x, y, ax, ay
 * hold the n movable positions and anchors; ax/ay may be NULL when
 * alpha <= 0. floor_x/floor_y are the minimum edge lengths (LinearSystems::
 * floorX/floorY). The systems stay on the device for ktg_solve. As a
 * by-product the HPWL of (x, y) is computed (ktg_build_hpwl). */
int ktg_build_b2b(ktg_ctx *ctx, const double *x, const double *y, double alpha,
                  const double *ax, const double *ay, double floor_x, double floor_y);

/* Kraftwerk2Placer::Impl::buildSystem (globalPlacer/kraftwerk2/
 * kraftwerk2_placer.cc:328-410) for both axes on the uploaded netlist (the
 * Kraftwerk2 Design's cells as the movable vertices, each fixed pin as a
 * fixed vertex at its fixedPosition with zero offset; nets may list a cell
 * more than once). with_rhs = withRhs. Kraftwerk2's rules: the high bound
 * pin is the last maximum, base = 2 w / (p - 1), edges to the row's own cell
 * are skipped, no anchor term, no diagonal floor. floor_x/floor_y are
 * Impl::floorX/floorY. The systems are then solved by ktg_solve, whose
 * per-axis iteration is Kraftwerk2's solve (kraftwerk2_placer.cc:86-126). */
int ktg_build_b2b_kraftwerk2(ktg_ctx *ctx, const double *x, const double *y, int with_rhs,
                             double floor_x, double floor_y);

/* Kraftwerk2's adjustments of the built systems: with move_weight (n values)
 * diag += move_weight and rhs = -move_weight * toward (kraftwerk2_placer.cc:
 * 716-721); then, when diag_floor > 0, diag = max(diag, diag_floor)
 * (kraftwerk2_placer.cc:433-437, floor 1e-12). move_weight may be NULL. */
int ktg_kraftwerk2_adjust(ktg_ctx *ctx, const double *move_weight, const double *toward_x,
                          const double *toward_y, double diag_floor);

/* LinearSystems::buildStar (simpl_lss.cc:116-201) for both axes: the star
 * model of SimPL's initial rounds, with a star variable after the movable
 * cells for every net of three or more pins that has a movable pin. *size
 * receives the number of rows (movable cells + stars); the systems stay on
 * the device for ktg_solve, bit-identical to the reference's. */
int ktg_build_star(ktg_ctx *ctx, int64_t *size);

/* HPWL of the positions given to the last ktg_build_b2b, equal to
 * simplPlacer::Impl::getHpwl on those positions (simpl_placer.cc:256-275).
 * Pointer mode applies to `out`. */
int ktg_build_hpwl(ktg_ctx *ctx, double *out);

/* Size of the system of one axis: n rows and nnz stored off-diagonal entries
 * (SparseSystem::size() and rowPtr.back(), simpl_lss.h:38-47). Host output;
 * synchronises the stream. */
int ktg_system_info(ktg_ctx *ctx, int axis, int64_t *n, int64_t *nnz);

/* Copies one axis system to host memory in SparseSystem's layout
 * (simpl_lss.h:38-43): row_ptr [n+1], col [nnz], val [nnz], diag [n],
 * rhs [n]. Any pointer may be NULL to skip it. */
int ktg_download_system(ktg_ctx *ctx, int axis, int64_t *row_ptr, int32_t *col, double *val,
                        double *diag, double *rhs);

/* Bound pins chosen for each net (the `extremes` of buildB2BAxis,
 * simpl_lss.cc:32-45): lo[k], hi[k] are pin indices inside net k. Host. */
int ktg_download_bound_pins(ktg_ctx *ctx, int axis, uint32_t *lo, uint32_t *hi);

/* Installs a caller-built system for one axis (host memory), for solving
 * systems assembled elsewhere (e.g. buildStar, simpl_lss.cc:116-201). The
 * other axis's system is kept when this one needs more room; a system of
 * another size than the other axis's invalidates that axis. */
int ktg_upload_system(ktg_ctx *ctx, int axis, int64_t n, const int64_t *row_ptr,
                      const int32_t *col, const double *val, const double *diag,
                      const double *rhs);

/* ---- PCG ------------------------------------------------------------------ */

/* solveBothAxes (simpl_lss.cc:203-290) on the current systems: FP64
 * Jacobi-PCG, x and y warm-started from and updated in place, stopping each
 * axis when its recursive relative residual ||r||/||b|| <= tol or after
 * max_iter steps, and deactivating an axis on non-positive p.Ap or r.z.
 * hist_x/hist_y (may be NULL) receive the residuals after each loop
 * iteration, as the IterateObserver sees them (capacity hist_cap).
 * Pointer mode applies to x, y, info, hist_x, hist_y. */
int ktg_solve(ktg_ctx *ctx, double *x, double *y, double tol, int64_t max_iter,
              ktg_solve_info *info, double *hist_x, double *hist_y, int64_t hist_cap);

/* Result of ktg_solve_mixed. resid_* is the true relative residual
 * ||b - A x|| / ||b|| in FP64 at exit. */
typedef struct {
    double resid_x;
    double resid_y;
    int64_t inner_x;               /* FP32 inner PCG iterations per axis       */
    int64_t inner_y;
    int32_t outer_x;               /* FP64 refinement rounds per axis          */
    int32_t outer_y;
    int32_t status;                /* KTG_OK or KTG_ERR_TIMEOUT                */
    int32_t stalled;               /* bit 0 / bit 1: x / y refinement stalled  */
    int64_t fp64_iters_x;          /* iterations of the FP64 fallback per axis */
    int64_t fp64_iters_y;
} ktg_mixed_info;

/* Mixed-precision variant of ktg_solve (no reference counterpart; the
 * reference solves in FP64 only, simpl_lss.cc:203-290): FP64 iterative
 * refinement around an FP32 Jacobi-PCG. Each round computes r = b - A x in
 * FP64, stops an axis once ||r|| / ||b|| <= tol (the true residual), and
 * otherwise solves A d = r with FP32 values and vectors (FP64 dot products
 * and alpha/beta) until the inner residual falls below inner_tol * ||r||,
 * then x += d. max_inner caps the FP32 iterations per axis (and the
 * iterations of the FP64 fallback below) and max_outer the rounds per axis. A round that does not halve the true residual marks the axis as
 * stalled; the solve is then finished by the FP64 kernel of ktg_solve from
 * the current x (in device pointer mode that FP64 pass always follows and
 * returns at once when both axes have converged). hist_x/hist_y receive the
 * true residual after each round. Pointer mode applies to x, y, info and
 * the histories. */
int ktg_solve_mixed(ktg_ctx *ctx, double *x, double *y, double tol, double inner_tol,
                    int64_t max_inner, int32_t max_outer, ktg_mixed_info *info,
                    double *hist_x, double *hist_y, int64_t hist_cap);

/* out = A in for the system of `axis` (0: x, 1: y) from the last build:
 * SparseSystem::multiply (simpl_lss.h:49-57). Each row sum starts from
 * diag * in and adds the row's entries in storage order, so out is
 * bit-identical to the reference's. Pointer mode applies to in and out
 * (n doubles each); in device mode the call is asynchronous on the
 * context's stream, and in and out must not overlap (other rows gather `in`
 * while `out` is written): an overlap returns KTG_ERR_ARG. */
int ktg_spmv(ktg_ctx *ctx, int32_t axis, const double *in, double *out);

/* ---- HPWL and density ---------------------------------------------------- */

/* simplPlacer::Impl::getHpwl (simpl_placer.cc:256-275). */
int ktg_hpwl(ktg_ctx *ctx, const double *x, const double *y, double *out);

/* Installs the bin grid used by ktg_occupancy (host memory). */
int ktg_set_grid(ktg_ctx *ctx, const ktg_grid_view *grid);

/* Impl::getOccupancy then Impl::getOverflow (simpl_placer.cc:282-297):
 * centre-binned movable area per bin (occ, [nx*ny], may be NULL) and the
 * scaled overflow. Bin sums are accumulated in 64-bit fixed point, so the map
 * is identical from run to run. */
int ktg_occupancy(ktg_ctx *ctx, const double *x, const double *y, double *occ,
                  double *overflow);

/* ---- look-ahead legalization ---------------------------------------------- */

/* Installs the free space, obstacles and die of LookAheadLegalizer
 * (globalPlacer/simpl/simpl_lal.h; FreeSpace of simpl_grid.h:130-232), host
 * memory, copied:
 *   row_y     [2*num_rows]  per row y start, y end; rows sorted by y start
 *   row_span  [num_rows+1]  row r's free spans are spans[row_span[r] ..
 *                           row_span[r+1]), row_span[0] = 0
 *   spans     [2*S]         x start, x end (spans already cut by the
 *                           obstacles, as FreeSpace::build leaves them)
 *   obstacles [4*num_obstacles]  lx ly ux uy of the fixed blocks
 *   die       [4]           lx ly ux uy
 * KTG_ERR_ARG on unsorted rows or a row_span that is not ascending. */
int ktg_set_free_space(ktg_ctx *ctx, int64_t num_rows, const double *row_y,
                       const int64_t *row_span, const double *spans, int64_t num_obstacles,
                       const double *obstacles, const double *die);

/* LookAheadLegalizer::legalize (globalPlacer/simpl/simpl_lal.cc:43-121, with
 * split :213-264, getStripes :266-312, nonlinearScale :314-363 and
 * clampToDie :365-372) in place
 * on x, y: overfilled clusters of the installed grid (ktg_set_grid, whose
 * density limit it uses) grown and legalized in batches by recursive
 * bisection with free-space-aware cutlines and stripe scaling, then clamped
 * to the die. Options as in simpl_options.h:24-26: maxLevel,
 * minCellsToSplit, stripeAreaFraction (defaults 20, 4, 0.1).
 * Positions are bit-identical to the reference when the cell areas are
 * multiples of 2^-s (s the occupancy's fixed-point shift; integer site
 * areas qualify): the bin occupancies it grows clusters from are exact then.
 * The cluster/grow/batch loop runs on the host between batches, so the call
 * synchronises with the context's stream and returns after the positions are
 * final in both pointer modes (device pointers are updated in place). */
int ktg_lal(ktg_ctx *ctx, double *x, double *y, int32_t max_level, int32_t min_cells_to_split,
            double stripe_area_fraction);

/* ---- batched solves ---------------------------------------------------------- */

/* Many independent systems (the x and y systems of many netlists, of uneven
 * sizes) solved in one persistent launch of thread-block clusters: one
 * cluster per system at a time, systems taken from a device work queue
 * largest first, captured once in a CUDA graph and replayed. Each system is
 * solved like ktg_solve (precision 0: FP64 Jacobi-PCG, recursive residual)
 * or like ktg_solve_mixed without the FP64 fallback (precision 1: FP32 PCG in
 * FP64 refinement, true residual; a stalled system reports status 1). No
 * reference counterpart: the reference solves one netlist at a time
 * (simpl_lss.cc:203-290). */
typedef struct ktg_batch ktg_batch;

typedef struct {
    int64_t iters;                 /* FP64 iterations, or FP32 inner ones      */
    int32_t outer;                 /* refinement rounds (precision 1)          */
    int32_t status;                /* KTG_OK, KTG_ERR_TIMEOUT, or 1 = stalled  */
    double resid;                  /* final relative residual                  */
    int64_t latency_ns;            /* device time from dequeue to done         */
} ktg_batch_result;

int ktg_batch_create(int device, ktg_batch **out);
void ktg_batch_destroy(ktg_batch *b);
const char *ktg_batch_last_error(const ktg_batch *b);
int ktg_batch_set_stream(ktg_batch *b, void *stream);
int64_t ktg_batch_size(const ktg_batch *b);
/* Appends one system (host CSR in SparseSystem's layout, start vector x0);
 * *id receives its index. */
int ktg_batch_add_system(ktg_batch *b, int64_t n, const int64_t *row_ptr, const int32_t *col,
                         const double *val, const double *diag, const double *rhs,
                         const double *x0, int64_t *id);
/* Appends the x and y systems a context built last (ids first, first+1);
 * x0/y0 are host start vectors. */
int ktg_batch_add_from_context(ktg_batch *b, ktg_ctx *ctx, const double *x0, const double *y0,
                               int64_t *first_id);
/* Cluster size (1, 2, 4, 8, 16 CTAs) and threads per CTA. */
int ktg_batch_set_shape(ktg_batch *b, int cluster, int threads);
int ktg_batch_get_shape(const ktg_batch *b, int *cluster, int *threads);
/* Times every launchable shape on this batch with an iteration cap of
 * probe_iter and keeps the fastest (the project autotuner). Resets x. */
int ktg_batch_autotune(ktg_batch *b, double tol, int precision, double inner_tol,
                       int64_t probe_iter, int *cluster, int *threads, float *best_ms);
/* Size classes: systems of at least `rows` rows (0 turns the split off) are
 * solved by a second persistent launch of `clusters` clusters of `cluster`
 * CTAs (1-16; 16 is a non-portable size) of `threads` threads, concurrent
 * with the launch of the batch shape over the rest, whose grid is cut to the
 * SMs left free. Each class drains its own work queue largest first. */
int ktg_batch_set_split(ktg_batch *b, int64_t rows, int cluster, int threads, int clusters);
/* The split in force and how many systems it puts in the large class (of the
 * systems left in the queues: offloaded pairs are in neither class). */
int ktg_batch_get_split(const ktg_batch *b, int64_t *rows, int *cluster, int *threads,
                        int *clusters, int *num_large);
/* Times full solves (iteration cap max_iter) with no split and with splits
 * that move the 1-16 largest queued systems to 16x1024, 8x1024 or 16x512
 * clusters (1-8 of them), and keeps the fastest; run it after
 * ktg_batch_autotune and ktg_batch_autotune_offload. *base_ms: the unsplit
 * time, *best_ms: the kept one (both 0 when every system is offloaded).
 * Resets x. */
int ktg_batch_autotune_split(ktg_batch *b, double tol, int precision, double inner_tol,
                             int64_t max_iter, float *base_ms, float *best_ms);
/* Whole-GPU path for the largest systems: pairs of consecutive systems of
 * equal size >= `rows` (the x and y systems of one netlist, as
 * ktg_batch_add_from_context adds them; 0 turns it off) are solved one pair
 * after another by an internal context on the whole GPU, before the cluster
 * launches take the rest: with precision 1 the mixed solve with
 * preconditioner `precond` (0 Jacobi, 2 aggregation) and coarse vector
 * `coarse` (0 none, 1 constant, 2 coupling share), with precision 0 the FP64
 * solve. Their results carry the mixed inner iterations and rounds (or the
 * FP64 iterations), the final true residual, status 1 when it misses tol,
 * and the latency from the pair's start. */
int ktg_batch_set_offload(ktg_batch *b, int64_t rows, int precond, int coarse);
/* The threshold in force and how many pairs it sends to the whole GPU. */
int ktg_batch_get_offload(const ktg_batch *b, int64_t *rows, int *pairs);
/* Times full solves with no offload and with the 2-64 largest systems
 * offloaded (split off during the trials, restored after) and keeps the
 * fastest; run it before ktg_batch_autotune_split. Resets x. */
int ktg_batch_autotune_offload(ktg_batch *b, double tol, int precision, double inner_tol,
                               int64_t max_iter, float *base_ms, float *best_ms);
/* Restores every system's start vector. */
int ktg_batch_reset_x(ktg_batch *b);
/* Enqueues the solve of every system on the batch's stream (graph replay). */
int ktg_batch_solve(ktg_batch *b, double tol, int64_t max_iter, int precision, double inner_tol);
/* Per-system results ([ktg_batch_size]); synchronises the stream. */
int ktg_batch_results(ktg_batch *b, ktg_batch_result *out);
int ktg_batch_get_x(ktg_batch *b, int64_t id, double *x);
int64_t ktg_batch_launch_count(const ktg_batch *b);

/* ---- learned preconditioner ------------------------------------------------ */

/* A learned sparse approximate inverse for ktg_solve_mixed (no reference
 * counterpart; the reference uses Jacobi only, simpl_lss.cc:203-290):
 *   M = D^-1/2 (I + S) D^-1/2,  s_e = t_e |a_e| / sqrt(d_i d_j),
 *   t_e = clamp(tanh(<p_i, p_j> / 4), -0.999, 0.999)
 * on A's own pattern (SPD for any network output on diagonally dominant
 * M-matrices such as the B2B systems, since rho(S) < 1),
 * where p comes from a 3-layer message-passing network over the cell-net
 * graph (hidden 64, BF16 tensor-core dense layers, FP32 accumulation).
 * Training minimises mean ||M A v - v||^2 / n over Rademacher probes v. */
typedef struct ktg_learned ktg_learned;

int64_t ktg_learned_num_params(void);
int ktg_learned_create(int device, uint64_t seed, ktg_learned **out);
void ktg_learned_destroy(ktg_learned *h);
const char *ktg_learned_last_error(const ktg_learned *h);
/* "tensor_cores" (2: BF16 tcgen05.mma with the accumulator in tensor memory,
 * the default; 1: BF16 mma.sync; 0: FP32 CUDA cores), "tc_ctas" (cap on the
 * tcgen05 layers' persistent CTAs, each walking 128-row tiles; 0 = four per
 * SM), "lr", "probes", "clip". */
int ktg_learned_set_option(ktg_learned *h, const char *key, double value);
/* FP32 parameters in the layout of oracle/learned_ref.py (host memory). */
int ktg_learned_get_params(ktg_learned *h, float *out);
int ktg_learned_set_params(ktg_learned *h, const float *in);
/* Loss and parameter gradient on the current B2B system of one axis of ctx
 * (probe seed `seed`); grad may be NULL. */
int ktg_learned_loss_grad(ktg_learned *h, ktg_ctx *ctx, int axis, uint64_t seed, double *loss,
                          float *grad);
/* One Adam step (global-norm clipped) on that system. */
int ktg_learned_train_step(ktg_learned *h, ktg_ctx *ctx, int axis, uint64_t seed, double *loss);
/* Computes M for both axes of ctx's current systems; ktg_solve_mixed uses it
 * when ktg_set_option(ctx, "precond", 1). A new build invalidates it. */
int ktg_learned_prepare(ktg_learned *h, ktg_ctx *ctx);
int64_t ktg_learned_launch_count(const ktg_learned *h);

/* The learned coarse vector of the two-level aggregation preconditioner
 * (ktg_download_coarse, "coarse" = 3; no reference counterpart). The same
 * 3-layer network runs once per netlist on features of the netlist alone
 * (pins per cell, sizes of its nets, fixed pins on them, area), giving an
 * embedding p (16 per cell) that is reused for every system of that
 * netlist; a per-system head (one hidden layer of 16, FP32) maps
 * (p_i, sum_j |a_ij| / a_ii, log a_ii - mean log a) to z_i = softplus(.) > 0.
 * An untrained head gives z = 1, the constant coarse vector.
 * Training minimises, over test vectors e_t of a system (the errors that the
 * aggregation-preconditioned CG leaves after a few iterations of a SimPL
 * solve), the share of their A-energy outside span(z):
 *   L = mean_t (1 - (z^T A e_t)^2 / ((z^T A z)(e_t^T A e_t))).
 * ktg_learned_coarse_loss_grad: loss and parameter gradient on axis `axis`
 * of ctx's current systems; e holds num_vec (1..4) host vectors of n
 * doubles. ktg_learned_coarse_train_step: the same, then one clipped Adam
 * step. ktg_learned_prepare_coarse: computes z for both axes of ctx's
 * current systems on ctx's stream (the embedding is recomputed only when
 * the netlist or the parameters changed) for the next mixed solve with
 * "coarse" = 3; a new build invalidates it. */
int ktg_learned_coarse_loss_grad(ktg_learned *h, ktg_ctx *ctx, int axis, const double *e,
                                 int32_t num_vec, double *loss, float *grad);
int ktg_learned_coarse_train_step(ktg_learned *h, ktg_ctx *ctx, int axis, const double *e,
                                  int32_t num_vec, double *loss);
int ktg_learned_prepare_coarse(ktg_learned *h, ktg_ctx *ctx);

/* ---- aggregation preconditioner (no reference counterpart) ---------------
 * With ktg_set_option(ctx, "precond", 2), ktg_solve_mixed preconditions its
 * FP32 inner PCG with the exact inverses of A's diagonal blocks over
 * aggregates of at most 8 rows, found by three levels of pairwise handshake
 * matching on the strength -a_ij / sqrt(a_ii a_jj) with Galerkin coarsening.
 * The rows are renumbered so that each aggregate is contiguous and lies in
 * one thread block of the solve, which applies M from shared memory. The
 * aggregates are built on the device (no host synchronisation) at the first
 * mixed solve after each build or upload of the systems.
 *
 * ktg_download_aggregates builds them now if needed and copies out, for the
 * 2n rows of the combined system (x rows 0..n-1, y rows n..2n-1):
 *   order[k]   combined row placed at position k (x rows come first),
 *   meta[k]    (first position of k's aggregate within its axis) * 8 +
 *              (aggregate size - 1),
 *   minv[8k+j] row k of its aggregate's block inverse, column j (FP32,
 *              zero beyond the aggregate's size).
 * Any of the three pointers may be NULL. Host memory. */
int ktg_download_aggregates(ktg_ctx *ctx, int32_t *order, int32_t *meta, float *minv);

/* Coarse correction of the aggregation preconditioner (no reference
 * counterpart). With ktg_set_option(ctx, "coarse", m) for m > 0 the mixed
 * solve's preconditioner is the two-level additive
 *   M r = B^-1 r + z (z^T A z)^-1 z^T r   per axis,
 * B the aggregates' block diagonal and z one coarse vector per axis:
 *   m = 1  the constant vector (the rigid motion of all cells, the smooth
 *          error block Jacobi leaves on SimPL systems);
 *   m = 2  z_i = sum_j |a_ij| / a_ii, the share of the row coupled to other
 *          movable cells (cells held only by fixed pins and anchors do not
 *          take part in the rigid motion);
 *   m = 3  the learned coarse vector (ktg_learned_prepare_coarse).
 * M is SPD for any nonzero z. The solve adds the term with no extra grid
 * barrier: it gathers only the block part B^-1 r, forms A z c from a stored
 * A z, and carries z^T r by recurrence beside its dot products.
 * ktg_download_coarse builds the aggregates and the coarse vector if needed
 * and copies out, in the permuted row order of ktg_download_aggregates,
 * z[k] and (A z)[k] (FP32, [2n]) and einv[axis] = 1 / (z^T A z) (FP64, [2],
 * 0 when not positive). Any pointer may be NULL. Host memory. */
int ktg_download_coarse(ktg_ctx *ctx, float *z, float *az, double *einv);

/* Phase timestamps of the last mixed solve (no reference counterpart), for
 * profiling: with ktg_set_option(ctx, "mixed_trace", cap) for cap > 0 block
 * 0 of the Chronopoulos-Gear mixed kernel records up to cap words
 * tag << 56 | %globaltimer ns at its phase boundaries (0 entry, 1 prologue
 * done, 2 refinement round start, 3 round residual reduced, 4 inner SpMV and
 * partials done, 5 scalars reduced, 6 inner iteration done, 7 exit); 0 turns
 * it off. ktg_download_mixed_trace copies min(cap, capacity) words to host
 * memory (unused words are 0). */
int ktg_download_mixed_trace(ktg_ctx *ctx, uint64_t *out, int64_t cap);

/* ---- Bookshelf reader ----------------------------------------------------
 * Reads a Bookshelf design directory <dir>/<name>.{nodes,wts,nets,pl,scl}
 * (name = the directory's own name, ".gz" variants read through zlib) with
 * the rules of BookshelfInputAdapter (adaptor/bookshelfToKTAdaptor.cc:137-672)
 * and flattens it like buildSimplDM (globalPlacer/simpl/simpl_dm.cc:16-85,
 * 262-279; die as getPlacementDieBox, datamodel/kt_die.cc:45-105). Host code;
 * line parsing on `threads` host threads (0 = all). The netlist view points
 * into the reader's arrays (valid until ktg_bookshelf_free) and goes straight
 * to ktg_upload_netlist. Status codes as elsewhere; the message of a failed
 * read is ktg_bookshelf_last_error() (per calling thread). */
typedef struct ktg_bookshelf ktg_bookshelf;

int ktg_bookshelf_read(const char *dir, int threads, ktg_bookshelf **out);
void ktg_bookshelf_free(ktg_bookshelf *b);
const char *ktg_bookshelf_last_error(void);
/* sizes[9]: vertices, movable, nets, pins, movable pins, fixed cells,
 * obstacles, rows, subrows. */
int ktg_bookshelf_sizes(const ktg_bookshelf *b, int64_t *sizes);
int ktg_bookshelf_view(const ktg_bookshelf *b, ktg_netlist_view *view);
/* Wall milliseconds of the read's phases (the reference times each file the
 * same way): ms[6] = nodes, wts, nets, pl, scl, flattening. */
int ktg_bookshelf_times(const ktg_bookshelf *b, double *ms);
/* die4 = (lx, ly, ux, uy); obstacles [K*4] (lx, ly, ux, uy) of the fixed
 * cells with area; rows [R*5] (coordinate, height, pitch, first subrow's xlo,
 * last subrow's xhi); subrows [S*3] (row index, xlo, xhi). NULL skips. */
int ktg_bookshelf_geometry(const ktg_bookshelf *b, double *die4, double *obstacles, double *rows,
                           double *subrows);

/* ---- tuning and introspection ------------------------------------------- */

/* Sets a kernel-shape option of this context (no reference counterpart; the
 * values are what the project autotuner chooses between):
 *   "pcg_lanes"  SpMV shape in the PCG: 32 = warp tiles (each warp streams
 *                the nonzeros of its range of rows 32 rows at a time, each
 *                lane adding its row's products in storage order; the ranges
 *                are balanced by nonzeros), 1 = one thread per row (the same
 *                row sums: the same solve bit for bit in form 2, to rounding
 *                in the others), 4 = four lanes per row; 0 = default (32)
 *   "pcg_form"   0: textbook PCG (three grid barriers per iteration),
 *                1: Chronopoulos-Gear form (two),
 *                3: textbook PCG with A p = A z + beta A p_prev by recurrence
 *                (two barriers; the same iterates to rounding), -1 = default
 *                (3),
 *                2: textbook PCG with every dot product summed in the
 *                reference's order (getDeterministicSum, simpl_parallel.h:
 *                35-51: 4,096-element chunks left to right, then the chunk
 *                sums in order): solutions, iteration counts and residual
 *                histories are bit-identical to solveBothAxes (about 3x the
 *                time of form 3)
 *   "agg_reuse"  K >= 0 (default 0): with the aggregation preconditioner, up
 *                to K builds in a row of the same netlist keep the last full
 *                build's aggregates and row order and only take the new
 *                values (permuted system, block inverses, coarse vector),
 *                skipping the matching and coarsening; the next build after
 *                K such builds, or after a new netlist, rebuilds everything.
 *                For SimPL's sequence of systems (one build per global
 *                iteration), whose couplings change little between builds.
 *   "hpwl_order" ktg_hpwl's sum of the (exact) per-net terms: 0 (default)
 *                a block tree; 2 the reference's getDeterministicSum order
 *                (simpl_parallel.h:35-51: chunks of 4,096 nets summed left to
 *                right, then the chunk sums in order), bit-identical to
 *                simplPlacer::Impl::getHpwl
 *   "precond"    0: Jacobi, 1: learned M (after ktg_learned_prepare),
 *                2: aggregation block-Jacobi, in ktg_solve_mixed
 *   "mixed_form" 1 (default): Chronopoulos-Gear mixed solve with per-block
 *                shared-memory slices; 0: textbook mixed solve
 *   "lal_subtree_cells"  ktg_lal: blocks of at most this many cells (0 to
 *                2048, default 2048) finish their bisection in one CTA;
 *                larger ones go level by level (0: always level by level).
 *                Results are identical either way.
 *   "lal_exact_sums"  ktg_lal: 1 (default) reads the area sums of split and
 *                nonlinearScale off integer prefix sums when every cell area
 *                is a multiple of 2^-q with the total below 2^52 (so the
 *                reference's sequential double sums are exact); 0 always
 *                sums sequentially in the reference's order.
 * Returns KTG_ERR_ARG for an unknown key or value. */
int ktg_set_option(ktg_ctx *ctx, const char *key, int64_t value);

/* Number of kernels this context has launched since creation (all entry
 * points). */
int64_t ktg_launch_count(const ktg_ctx *ctx);

/* Counters of the last ktg_lal call, up to `count` (at most 16) of:
 * batches, regions, bisection rounds (one-CTA launches and level-by-level
 * levels, summed over batches), host synchronisations, blocks (summed over
 * rounds), ms in the batches' bisection, ms in the occupancy refreshes, ms
 * in total, ms in the one-CTA subtree launches, level-by-level levels,
 * one-CTA blocks, one-CTA blocks handed back, and of those the ones with too
 * many cells or obstacles, too many sub-blocks at one level, a full sort
 * buffer, full stripe storage (host wall clock). No reference
 * counterpart. */
int ktg_lal_stats(ktg_ctx *ctx, double *out, int32_t count);

/* Test of the bounded device waits: a cooperative launch in which one block
 * never arrives at a grid barrier, so the other's wait gives up after
 * timeout_ns (at most 1 s) and reports through the status word; run once
 * with each of the library's two grid barriers. *status_out receives
 * KTG_ERR_TIMEOUT when both gave up as they should, else the first other
 * status. Nothing faults and the context stays usable. No reference
 * counterpart (the reference has no device). */
int ktg_selftest_wait_timeout(ktg_ctx *ctx, int64_t timeout_ns, int *status_out);

/* ---- allocation-free HPWL ------------------------------------------------ */

/* Largest net count ktg_hpwl_noalloc accepts. */
#define KTG_NOALLOC_HPWL_MAX_NETS 4194304

/* HPWL of the movable positions (x, y), like ktg_hpwl, for callers that may
 * not allocate GPU memory: code running where cudaMalloc is forbidden or
 * unsafe (inside a host callback, under a memory pool or allocator owned by
 * another runtime, in a service with a fixed memory budget). It has no
 * counterpart in the reference, which never allocates device memory at all.
 *
 * Nothing is allocated or freed, and no context is needed: every argument is
 * a device pointer on the current device (netlist arrays as in
 * ktg_netlist_view, with 32-bit net_start), `out` receives one double, and
 * the work is enqueued on `stream` (a cudaStream_t, NULL = legacy default).
 * The reduction's scratch (one partial per 256 nets plus a ticket, about
 * 128 KiB) is a static device array that every GPU which loads this library
 * holds until the process exits. Limits and caveats:
 *   - num_nets above KTG_NOALLOC_HPWL_MAX_NETS returns KTG_ERR_RANGE;
 *   - the first call made with a given CUDA context current looks up the
 *     scratch array's address in that context (cudaGetSymbolAddress) and
 *     keeps it under the context's id, so make that first call before any
 *     stream capture begins; a context created later (another driver
 *     context, or the primary one again after cudaDeviceReset) gets its own
 *     lookup, never a stale address;
 *   - all calls share the one scratch array: calls that overlap on the GPU
 *     (different streams, or host threads without ordering) race and give
 *     wrong sums. Serialise them on one stream.
 * Returns KTG_OK or a negative KTG_ERR_* code. */
int ktg_hpwl_noalloc(const int32_t *net_start, const int32_t *pin_cell,
                     const int32_t *var_of_vertex, const double *off_x, const double *off_y,
                     const double *fixed_x, const double *fixed_y, const double *x,
                     const double *y, int64_t num_nets, double *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* KTPLACE_B200_H */
