// Allocation-free HPWL entry point (sm_100a).
//
// Some callers cannot allocate device memory at all: code that runs inside a
// host callback or a memory-pool-restricted service, or a caller whose
// allocator is owned by another runtime and must not see cudaMalloc/cudaFree
// calls behind its back. ktg_hpwl_noalloc serves them: the caller passes every
// input and the output as device pointers, and the only scratch the
// reduction needs (one partial sum per block plus a completion ticket) lives
// in a file-scope __device__ array that exists on every GPU that loads this
// library, until the process exits. No context is created and nothing is
// allocated or freed.
//
// The per-net term is the half perimeter of simplPlacer::Impl::getHpwl
// (globalPlacer/simpl/simpl_placer.cc:256-275); the sum is a fixed-shape tree,
// so the result equals ktg_hpwl on the same positions.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "ktg_common.cuh"
#include "ktplace_b200.h"

namespace {

constexpr int kThreads = 256;
// Maximum blocks of one call: 16384 blocks x 256 threads = 4,194,304 nets.
constexpr int kMaxBlocks = KTG_NOALLOC_HPWL_MAX_NETS / kThreads;
// Element 0 holds the completion ticket (as a 32-bit word), elements 32..
// the per-block partial sums: 128 KiB + 256 B in all.
constexpr int kTicketSlots = 32;

static __device__ __align__(256) double g_hpwl_scratch[kTicketSlots + kMaxBlocks];

// Looked-up scratch addresses, one per CUDA context. A context is named by
// its process-unique id (cuCtxGetId), never by its handle or by the device
// ordinal alone: after a context is destroyed (cudaDeviceReset, or a driver
// context the caller made current and later destroyed) a new context may get
// the same handle and the same ordinal, but this library's module, and so
// the scratch array, is loaded into it afresh at a possibly different
// address. The ids of destroyed contexts are never reused, so a stale entry
// is never matched.
struct ScratchEntry {
    unsigned long long ctx_id;
    double *addr;
};
constexpr int kCacheSize = 64;
std::mutex g_setup_mutex;
ScratchEntry g_cache[kCacheSize] = {};
int g_cache_next = 0;

typedef int (*CtxGetCurrentFn)(void **);
typedef int (*CtxGetIdFn)(void *, unsigned long long *);
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;
bool g_driver_looked_up = false;

__global__ void __launch_bounds__(kThreads)
    k_hpwl_noalloc(const int32_t *__restrict__ net_start, const int32_t *__restrict__ pin_cell,
                   const int32_t *__restrict__ var_of_vertex, const double *__restrict__ off_x,
                   const double *__restrict__ off_y, const double *__restrict__ fixed_x,
                   const double *__restrict__ fixed_y, const double *__restrict__ x,
                   const double *__restrict__ y, int32_t num_nets, double *__restrict__ scratch,
                   double *__restrict__ out) {
    __shared__ double red[40];
    unsigned *ticket = reinterpret_cast<unsigned *>(scratch);
    double *partials = scratch + kTicketSlots;
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    double term = 0.0;
    if (k < num_nets) {
        const int32_t s = net_start[k];
        const int32_t e = net_start[k + 1];
        double bx0 = __longlong_as_double(0x7ff0000000000000ll);  // +inf
        double by0 = bx0;
        double bx1 = -bx0;
        double by1 = -bx0;
        for (int32_t p = s; p < e; ++p) {
            const int32_t cell = pin_cell[p];
            const int32_t var = var_of_vertex[cell];
            const double px = (var >= 0 ? x[var] : fixed_x[cell]) + off_x[p];
            const double py = (var >= 0 ? y[var] : fixed_y[cell]) + off_y[p];
            bx0 = ktg::ref_min(bx0, px);
            by0 = ktg::ref_min(by0, py);
            bx1 = ktg::ref_max(bx1, px);
            by1 = ktg::ref_max(by1, py);
        }
        if (e - s >= 2 && !(bx0 > bx1 || by0 > by1)) term = (bx1 - bx0) + (by1 - by0);
    }
    const double bs = ktg::block_sum(term, red);
    if (threadIdx.x == 0) __stcg(partials + blockIdx.x, bs);
    if (ktg::last_block_done(ticket)) {
        const double total = ktg::sum_partials(partials, gridDim.x, red);
        if (threadIdx.x == 0) *out = total;
    }
}

// Address of the scratch array in the current context, looked up with
// cudaGetSymbolAddress on the first call made with that context current and
// cached under the context's id. When no context is current yet (the
// runtime creates the device's primary context during the lookup) or the
// driver cannot name contexts (no cuCtxGetId), nothing is cached and the
// address is looked up again on the next call.
int scratch_for_current_context(double **addr) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return KTG_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_driver_looked_up) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_id = reinterpret_cast<CtxGetIdFn>(f);
        g_driver_looked_up = true;
    }
    unsigned long long id = 0;
    void *ctx = nullptr;
    const bool named = g_ctx_current && g_ctx_id && g_ctx_current(&ctx) == 0 && ctx &&
                       g_ctx_id(ctx, &id) == 0;
    if (named) {
        for (const ScratchEntry &e : g_cache)
            if (e.addr && e.ctx_id == id) {
                *addr = e.addr;
                return KTG_OK;
            }
    }
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_hpwl_scratch) != cudaSuccess || p == nullptr)
        return KTG_ERR_CUDA;
    if (named) {
        g_cache[g_cache_next] = ScratchEntry{id, static_cast<double *>(p)};
        g_cache_next = (g_cache_next + 1) % kCacheSize;
    }
    *addr = static_cast<double *>(p);
    return KTG_OK;
}

}  // namespace

extern "C" int ktg_hpwl_noalloc(const int32_t *net_start, const int32_t *pin_cell,
                                const int32_t *var_of_vertex, const double *off_x,
                                const double *off_y, const double *fixed_x, const double *fixed_y,
                                const double *x, const double *y, int64_t num_nets, double *out,
                                void *stream) {
    if (num_nets < 0 || out == nullptr || net_start == nullptr) return KTG_ERR_ARG;
    if (num_nets > KTG_NOALLOC_HPWL_MAX_NETS) return KTG_ERR_RANGE;
    if (num_nets > 0 && (!pin_cell || !var_of_vertex || !off_x || !off_y || !fixed_x ||
                         !fixed_y || !x || !y))
        return KTG_ERR_ARG;
    double *scratch = nullptr;
    int rc = scratch_for_current_context(&scratch);
    if (rc != KTG_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The ticket must start at zero; the partials are always written before
    // they are read.
    if (cudaMemsetAsync(scratch, 0, sizeof(double), st) != cudaSuccess) return KTG_ERR_CUDA;
    const int blocks = num_nets > 0 ? static_cast<int>((num_nets + kThreads - 1) / kThreads) : 1;
    k_hpwl_noalloc<<<blocks, kThreads, 0, st>>>(net_start, pin_cell, var_of_vertex, off_x, off_y,
                                                fixed_x, fixed_y, x, y,
                                                static_cast<int32_t>(num_nets), scratch, out);
    return cudaGetLastError() == cudaSuccess ? KTG_OK : KTG_ERR_CUDA;
}
