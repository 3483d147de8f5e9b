// Buffers of the aggregation preconditioner (built by ktg_agg.cu, read by
// the mixed-precision solve).
#pragma once

#include <cstdint>
#include <vector_types.h>

namespace ktg {

struct AggState {
    int64_t cap_rows = 0;  // 2n capacity
    int64_t cap_nnz = 0;   // nnz(x) + nnz(y) capacity
    int grid_cap = 0;
    // level work: per node of the current level (mate, pick, flag, cid,
    // sizes, members by position), per fine row (its node in cur / cur2,
    // position, best candidate, internal sum, its node's diagonal dc), per
    // fine entry (strength sbuf and neighbour node bbuf of the level)
    int32_t *mate = nullptr, *pick = nullptr, *flag = nullptr, *cid = nullptr;
    int32_t *size_a = nullptr, *size_b = nullptr;
    int32_t *cur = nullptr, *cur2 = nullptr, *pos = nullptr;
    int32_t *mem = nullptr;        // [4 * 2n] members of a node by position
    int32_t *cand_b = nullptr;     // [2n]
    double *cand_s = nullptr;      // [2n]
    double *tbuf = nullptr;        // [2n]
    double *dc = nullptr;          // [2n]
    double *sbuf = nullptr;        // [nnz]
    int32_t *bbuf = nullptr;       // [nnz]
    int32_t *counts = nullptr;     // [8] node counts per level, totals
    int32_t *tile_sum = nullptr;   // scan tiles
    int64_t tiles_cap = 0;
    // result
    int32_t *agg_start = nullptr;  // [2n + 1]
    int32_t *order = nullptr, *newpos = nullptr;  // [2n]
    int32_t *prp = nullptr;        // [2n + 1] combined offsets
    int32_t *pcol = nullptr;       // [nnz] per-axis local columns
    double *pval = nullptr;        // [nnz]
    float *pval32 = nullptr;       // [nnz]
    double *pdiag = nullptr, *prhs = nullptr, *px = nullptr;  // [2n]
    float *minv = nullptr;         // [2n * 8]
    int32_t *meta = nullptr;       // [2n] per-axis first * 8 + size - 1
    int32_t *blk_start = nullptr;  // [grid + 1]
    double *gslice = nullptr;      // per-block slices when shared memory is too small
    int64_t gslice_cap = 0;
    int blk_grid = 0;              // grid the blk_start array was built for
    // coarse correction (the mixed solve's u = B^-1 r + z c): per permuted row
    // (z, (A z)) in FP32, per axis 1 / (z^T A z) (0: no correction)
    float2 *zaz = nullptr;         // [2n]
    double *zd = nullptr;          // [2n] z in FP64 (the SpMV's input)
    int z_mode = 0;                // mode whose z is in zd (0: none)
    // aggregate structure of the last full build: sizes buffer, rows and
    // netlist it belongs to, later builds that reused it
    const int32_t *final_size = nullptr;
    int64_t struct_rows = -1;
    int64_t struct_gen = -1;
    int builds_on_struct = 0;
    int64_t z_gen = -1;            // learned coarse vector generation in zd (mode 3)
    double *coarse_einv = nullptr; // [2]
    double *coarse_part = nullptr; // [2 * blocks] per-block z^T A z
    unsigned *ticket = nullptr;    // last-block ticket of the coarse set-up
    int coarse_mode = 0;           // mode the zaz array holds (0: none built)
};

}  // namespace ktg
