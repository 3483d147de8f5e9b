// Self-test of the bounded device waits (sm_100a).
//
// Every grid barrier in this library gives up after a %globaltimer deadline
// and reports KTG_ERR_TIMEOUT through a status word instead of hanging.
// ktg_selftest_wait_timeout exercises exactly that path on purpose, without
// faulting anything: a two-block cooperative launch in which block 1 returns
// at once and never arrives, so block 0's wait runs out after `timeout_ns`,
// writes the status and returns; once with grid_barrier and once with
// grid_sync. The context stays usable afterwards.
#include <cuda_runtime.h>

#include "ktg_common.cuh"
#include "ktg_context.h"
#include "ktplace_b200.h"

namespace ktg {
namespace {

// form 0: grid_barrier; form 1: grid_sync (the persistent solvers' barrier)
__global__ void k_wait_for_absent_block(unsigned *count, unsigned *gen, int *status,
                                        uint64_t timeout_ns, int form) {
    if (blockIdx.x == 1) return;  // never arrives
    if (form == 0) {
        grid_barrier(count, gen, status, global_timer_ns() + timeout_ns);
    } else {
        GridSync g = grid_sync_init(count, gen, status);
        grid_sync(g, global_timer_ns() + timeout_ns);
    }
}

}  // namespace
}  // namespace ktg

extern "C" int ktg_selftest_wait_timeout(ktg_ctx *c, int64_t timeout_ns, int *status_out) {
    if (!c || timeout_ns <= 0 || timeout_ns > 1000000000ll || !status_out) return KTG_ERR_ARG;
    KTG_CUDA(c, cudaSetDevice(c->device));
    unsigned *count = c->counters + 2, *gen = c->counters + 3;
    int *status = c->status;
    uint64_t t = static_cast<uint64_t>(timeout_ns);
    // both barrier forms must give up with KTG_ERR_TIMEOUT; the first status
    // that is not a timeout is reported
    int seen = 0;
    for (int form = 0; form < 2; ++form) {
        KTG_CUDA(c, cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
        KTG_CUDA(c, cudaMemsetAsync(c->counters + 2, 0, sizeof(unsigned), c->stream));
        void *args[] = {&count, &gen, &status, &t, &form};
        KTG_CUDA(c, cudaLaunchCooperativeKernel((void *)ktg::k_wait_for_absent_block, dim3(2),
                                                dim3(32), args, 0, c->stream));
        ++c->launches;
        KTG_CUDA(c, cudaMemcpyAsync(c->h_status, c->status, sizeof(int), cudaMemcpyDeviceToHost,
                                    c->stream));
        KTG_CUDA(c, cudaStreamSynchronize(c->stream));
        if (form == 0 || seen == KTG_ERR_TIMEOUT) seen = *c->h_status;
    }
    *status_out = seen;
    // leave the barrier words clean for the next solve
    KTG_CUDA(c, cudaMemsetAsync(c->counters + 2, 0, sizeof(unsigned), c->stream));
    KTG_CUDA(c, cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
    KTG_CUDA(c, cudaStreamSynchronize(c->stream));
    return KTG_OK;
}
