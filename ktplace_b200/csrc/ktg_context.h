// Host-side context of the ktplace_b200 C ABI.
//
// Device layout (all device-resident for the life of a netlist):
//   netlist  : var_of_vertex[V] i32, fixed_x/y[V] f64,
//              net_start[N+1] i32, pin_cell/pin_var[P] i32, off_x/off_y[P] f64,
//              net_base[N] f64 (= weight / (degree - 1)), net_mov[N] i32,
//              pin_start[n+1] i32, pin_ref[Pm] int2 (net, pin),
//              width/height/area[n] f64
//   systems  : per axis row_ptr[n+1] i32, col[cap] i32, val[cap] f64,
//              diag[n], rhs[n] f64, bound pins lo/hi[N] u32
//   PCG      : per axis r, z, p, ap [n] f64, positions x/y, anchors [n] f64
//   density  : occ_fx[bins] i64 fixed point, avail[bins] f64
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "ktplace_b200.h"

namespace ktg {

// Bits of ktg_ctx::attr_bits.
constexpr unsigned kAttrOccupancy = 1u;  // k_occ_accum<true> opt-in shared memory
constexpr unsigned kAttrMixed = 2u;      // k_pcg_mixed_cg opt-in shared memory

struct AggState;  // aggregation preconditioner buffers (ktg_agg.cu)
struct LalState;  // free space and scratch of the look-ahead legalizer (ktg_lal.cu)

struct AxisSystem {
    int32_t *row_ptr = nullptr;  // [n+1]
    int32_t *col = nullptr;      // [cap]
    double *val = nullptr;       // [cap]
    double *diag = nullptr;      // [n]
    double *rhs = nullptr;       // [n]
    uint32_t *lo = nullptr;      // [N]
    uint32_t *hi = nullptr;      // [N]
    double *r = nullptr, *z = nullptr, *p = nullptr, *ap = nullptr, *s = nullptr;  // [n]
    // mixed precision: FP32 copy of val and the inner vectors
    float *val32 = nullptr;                                                 // [cap]
    float *d32 = nullptr, *r32 = nullptr, *z32 = nullptr, *p32 = nullptr, *ap32 = nullptr;  // [n]
    // learned preconditioner: S values on A's pattern and D^-1/2 r scratch
    float *s32 = nullptr;   // [cap]
    float *rs32 = nullptr;  // [n]
};

}  // namespace ktg

struct ktg_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int ptr_mode = KTG_PTR_HOST;
    std::string err;
    int64_t launches = 0;
    int pcg_lanes = 0;  // 0: library default; 32 warp tiles, 1 or 4 lanes per row in the PCG SpMV
    int pcg_form = -1;  // -1: library default; 0 textbook PCG, 1 Chronopoulos-Gear,
                        // 2 textbook PCG in the reference's summation order,
                        // 3 textbook PCG with A p by recurrence
    double *exact_prod = nullptr;   // form 2: products of the dots [3 * 2n]
    double *exact_cpart = nullptr;  // form 2: chunk sums [6 * chunks]
    int64_t exact_prod_cap = 0, exact_cpart_cap = 0;
    int mixed_form = 1; // mixed solve: 0 textbook (global vectors), 1 Chronopoulos-Gear
    // Per-device launch set-up, done once per context (a context owns one
    // device): opt-in shared memory attributes set (kAttr* bits and the PCG
    // variants' bits), the PCG's shared-memory budgets and ktg_spmv's blocks
    // per SM.
    unsigned attr_bits = 0;
    unsigned pcg_attr_bits = 0;
    size_t pcg_smem_budget[4][3] = {};
    int spmv_per_sm = 0;

    // netlist sizes
    bool have_netlist = false;
    int64_t V = 0, n = 0, N = 0, P = 0, Pm = 0;
    int64_t cap_nnz = 0;  // col/val capacity per axis (upper bound on nnz)
    double fx_scale = 1.0;
    int area_shift = -1;  // areas are multiples of 2^-area_shift with exact sums (-1: not)

    // netlist arrays
    int32_t *var_of_vertex = nullptr;
    double *fixed_x = nullptr, *fixed_y = nullptr;
    int32_t *net_start = nullptr, *pin_cell = nullptr, *pin_var = nullptr;
    double *off_x = nullptr, *off_y = nullptr, *net_base = nullptr, *net_weight = nullptr;
    int32_t *net_mov = nullptr;
    int32_t *pin_start = nullptr;
    int2 *pin_ref = nullptr;
    double *width = nullptr, *height = nullptr, *area = nullptr;

    // systems
    ktg::AxisSystem sys[2];
    bool have_system = false;  // both axes valid with sys_n rows
    bool axis_valid[2] = {false, false};
    bool val32_valid = false;  // sys[*].val32 mirrors sys[*].val
    bool precond_ready = false;  // sys[*].s32 holds learned values for the current systems
    int precond = 0;             // 0 Jacobi, 1 learned, 2 aggregation (ktg_set_option "precond")
    ktg::AggState *agg = nullptr;  // aggregation preconditioner of the current systems
    bool agg_ready = false;        // agg holds aggregates of the current systems
    int agg_reuse = 0;             // aggregation: builds that may reuse the last structure
    int coarse = 0;                // coarse vector of the aggregation solve: 0 none,
                                   // 1 constant, 2 coupling share, 3 learned
    // inputs of the learned coarse vector (coarse 3), evaluated per row by the
    // aggregation build: the head's parameters (a copy, ktg_coarse_head.cuh),
    // the trunk embedding below and each axis's mean log diagonal
    float *coarse_head_w = nullptr;   // [kCoarseHeadParams]
    double *coarse_logd = nullptr;    // [2]
    bool coarse_z_ready = false;      // those inputs belong to the current systems
    int64_t coarse_z_gen = 0;         // bumped whenever they are rewritten
    // trunk embedding of this context's netlist under one learned parameter
    // set (computed once per netlist, reused by every build's head pass)
    float *coarse_emb = nullptr;      // [n x 16]
    int64_t coarse_emb_cap = 0;
    uint64_t coarse_emb_owner = 0;    // id of the learned handle that wrote it
    int64_t coarse_emb_version = -1, coarse_emb_gen = -1;
    int64_t netlist_gen = 0;          // bumped by every ktg_upload_netlist
    const ktg_mixed_info *pcg_gate = nullptr;  // see PcgArgs::gate (ktg_pcg.cu)
    unsigned long long *mixed_trace = nullptr;  // phase stamps of the mixed solve (null: off)
    int hpwl_order = 0;               // 0 block tree, 2 the reference's chunked order
    double *hpwl_terms = nullptr;     // per-net terms for hpwl_order 2
    int64_t hpwl_terms_cap = 0;
    int32_t mixed_trace_cap = 0;
    int64_t sys_n = 0;        // rows of the current systems (n, or more after upload)
    int64_t sys_cap_n = 0;    // allocated rows for r/z/p/ap/diag/rhs
    int64_t sys_cap_nnz = 0;  // allocated entries for col/val

    // staging (host pointer mode) and scratch
    double *x = nullptr, *y = nullptr, *ax = nullptr, *ay = nullptr;  // [max(n, sys_cap_n)]
    int64_t stage_cap = 0;
    int32_t *row_cnt = nullptr;      // [2n]
    int32_t *heavy_rows = nullptr;   // [1 + 2n] B2B rows filled one warp each: count, rows
    int64_t *block_sum = nullptr;    // [2 * blocks]
    int64_t *nnz_dev = nullptr;      // [2]
    double *partials = nullptr;      // reduction partials
    int64_t partials_cap = 0;
    unsigned *counters = nullptr;    // [8] last-block tickets, barrier count/gen
    int *status = nullptr;           // [1]
    double *scalars = nullptr;       // [8] hpwl of build, hpwl, overflow, ...
    ktg_solve_info *info_dev = nullptr;
    ktg_mixed_info *minfo_dev = nullptr;
    ktg_mixed_info *h_minfo = nullptr;
    double *hist_dev = nullptr;      // [2 * hist_cap_dev]
    int64_t hist_cap_dev = 0;

    // host pinned mirrors for scalar results
    double *h_scalars = nullptr;     // [8]
    ktg_solve_info *h_info = nullptr;
    int64_t *h_nnz = nullptr;        // [2]
    int *h_status = nullptr;

    // density grid
    bool have_grid = false;
    int64_t nx = 0, ny = 0;
    double origin_x = 0, origin_y = 0, dx = 1, dy = 1, total_avail = 0, density_limit = 1;
    double *avail = nullptr;         // [bins]
    std::vector<double> avail_host;  // [bins] host copy (the legalizer's cluster loop)
    unsigned long long *occ_fx = nullptr;  // [bins] two's-complement fixed point
    double *occ = nullptr;           // [bins] staging for host mode
    int64_t bins_cap = 0;

    // look-ahead legalization
    ktg::LalState *lal = nullptr;
    bool have_free_space = false;
    int lal_subtree_cells = 2048;  // blocks up to this many cells finish in one CTA
    int lal_exact_sums = 1;        // area sums from integer prefixes when exact
};

namespace ktg {

// Launchers (one per kernel family), implemented in the .cu files. They
// enqueue on ctx->stream and return a KTG_* code.
int launch_build_b2b(ktg_ctx *ctx, const double *x, const double *y, double alpha,
                     const double *ax, const double *ay, double floor_x, double floor_y);
int launch_hpwl(ktg_ctx *ctx, const double *x, const double *y, double *out_dev);
int launch_spmv(ktg_ctx *ctx, int axis, const double *in, double *out);
int launch_build_kraftwerk2(ktg_ctx *ctx, const double *x, const double *y, bool with_rhs,
                            double floor_x, double floor_y);
int launch_kraftwerk2_adjust(ktg_ctx *ctx, const double *move_weight, const double *toward_x,
                             const double *toward_y, double diag_floor);
int launch_solve(ktg_ctx *ctx, double *x, double *y, double tol, int64_t max_iter,
                 ktg_solve_info *info_dev, double *hist_x, double *hist_y, int64_t hist_cap);
int launch_occupancy(ktg_ctx *ctx, const double *x, const double *y, double *occ_dev,
                     double *overflow_dev);
int launch_solve_mixed(ktg_ctx *ctx, double *x, double *y, double tol, double inner_tol,
                       int64_t max_inner, int32_t max_outer, ktg_mixed_info *info_dev,
                       double *hist_x, double *hist_y, int64_t hist_cap);

int build_star(ktg_ctx *ctx, int64_t *size_out, int (*reserve)(ktg_ctx *, int64_t, int64_t));
// Capacity for systems of `rows` rows and `nnz` entries per axis (growing
// keeps the installed systems).
int reserve_system_arrays(ktg_ctx *ctx, int64_t rows, int64_t nnz);
int load_system_device(ktg_ctx *ctx, int axis, int64_t n, int64_t m, const int32_t *rp,
                       const int32_t *col, const double *val, const double *diag,
                       const double *rhs);

// Aggregation preconditioner (ktg_agg.cu): build for the current systems,
// per-solve set-up (block row ranges, permuted positions) and write-back.
int build_agg(ktg_ctx *ctx);
int build_agg_values(ktg_ctx *ctx);
int prepare_agg(ktg_ctx *ctx);
int agg_prepare_solve(ktg_ctx *ctx, int grid, const double *x, const double *y, int32_t *rows_cap);
int agg_finish_solve(ktg_ctx *ctx, double *x, double *y);
double *agg_global_slices(ktg_ctx *ctx, int64_t doubles);
int agg_coarse_setup(ktg_ctx *ctx, int mode);
void free_agg(ktg_ctx *ctx);

// Look-ahead legalization (ktg_lal.cu): free space (host arrays) and the
// legalizer on device positions.
int set_free_space(ktg_ctx *ctx, int64_t nrows, const double *row_y, const int64_t *row_span,
                   const double *spans, int64_t nobst, const double *obst, const double *die4);
int launch_lal(ktg_ctx *ctx, double *x, double *y, int32_t max_level, int32_t min_cells,
               double stripe_fraction);
void free_lal(ktg_ctx *ctx);
int lal_stats(ktg_ctx *ctx, double *out, int count);

int set_error(ktg_ctx *ctx, int code, const std::string &msg);
int cuda_check(ktg_ctx *ctx, cudaError_t e, const char *what);

}  // namespace ktg

#define KTG_CUDA(ctx, call)                                           \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) return ktg::cuda_check((ctx), e_, #call); \
    } while (0)
