// Standalone SpMV of one assembled system (sm_100a): out = A in, where A is
// the diagonal plus the off-diagonal CSR of the last B2B (or Kraftwerk2, or
// star) build on one axis.
//
// Replaces SparseSystem::multiply (globalPlacer/simpl/simpl_lss.h:49-57):
// every row sum starts from diag * in and adds the row's entries in storage
// order, so the result is bit-identical to the reference's. The rows are
// cut into one even wave of blocks (at least kSpmvMinRows rows each); inside
// a block the warps take row ranges balanced by nonzeros and stream them as
// warp tiles (ktg_spmv.cuh). Unlike
// the persistent solvers, many blocks share an SM here, so the gathers of
// several blocks are in flight at once.
#include <algorithm>
#include <climits>

#include "ktg_common.cuh"
#include "ktg_context.h"
#include "ktg_spmv.cuh"

namespace ktg {
namespace {

constexpr int kSpmvThreads = 256;
constexpr int32_t kSpmvMinRows = 256;  // rows per block at least

__global__ void __launch_bounds__(kSpmvThreads)
    k_spmv(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
           const double *__restrict__ val, const double *__restrict__ diag,
           const double *__restrict__ in, double *__restrict__ out, int32_t n, int32_t rows) {
    __shared__ __align__(16) double tilebuf[(kSpmvThreads / 32) * kTileChunk];
    __shared__ int32_t wb[kSpmvThreads / 32 + 1];
    const int32_t r0 = static_cast<int32_t>(blockIdx.x) * rows;  // < n: grid covers n
    const int32_t R = min(rows, n - r0);
    const int64_t base = __ldg(rp + r0);
    warp_row_bounds(R, wb, [&](int32_t l) {
        return int64_t(__ldg(rp + r0 + l)) - base + int64_t(kRowCost) * l;
    });
    warp_tile_spmv<double>(
        r0, INT32_MAX, R, kAllAxes, wb, tilebuf,
        [&](int, const int32_t *&trp, const int32_t *&tcol, const double *&tval,
            const double *&tin) {
            trp = rp;
            tcol = col;
            tval = val;
            tin = in;
        },
        [&](int32_t, int, int32_t i) { return __ldg(diag + i) * __ldg(in + i); },
        [&](int32_t, int, int32_t i, double s) { out[i] = s; });
}

}  // namespace

int launch_spmv(ktg_ctx *c, int axis, const double *in, double *out) {
    const int32_t n = static_cast<int32_t>(c->sys_n);
    if (n == 0) return KTG_OK;
    const AxisSystem &s = c->sys[axis];
    // one even wave: as many blocks as fit on the GPU at once, each at least
    // kSpmvMinRows rows (several waves beyond that)
    int &per_sm = c->spmv_per_sm;  // once per context (one device)
    if (per_sm == 0) {
        KTG_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spmv, kSpmvThreads,
                                                                  0));
        if (per_sm < 1) per_sm = 1;
    }
    const int64_t slots = static_cast<int64_t>(per_sm) * c->num_sms;
    const int32_t rows = static_cast<int32_t>(
        std::max<int64_t>(kSpmvMinRows, (n + slots - 1) / slots));
    const int blocks = static_cast<int>((n + rows - 1) / rows);
    k_spmv<<<blocks, kSpmvThreads, 0, c->stream>>>(s.row_ptr, s.col, s.val, s.diag, in, out, n,
                                                   rows);
    ++c->launches;
    KTG_CUDA(c, cudaGetLastError());
    return KTG_OK;
}

}  // namespace ktg
