// Device helpers shared by the ktplace_b200 kernels (sm_100a).
//
// Everything here is deterministic: reductions use a fixed tree whose shape
// depends only on the launch configuration, never on timing, and waits are
// bounded by %globaltimer deadlines so a kernel can never hang its GPU.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ktg {

constexpr int kWarp = 32;

// std::max / std::min exactly as the reference's expressions evaluate them:
// max(a, b) = (a < b) ? b : a, min(a, b) = (b < a) ? b : a (NaN handling
// included).
__device__ __forceinline__ double ref_max(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double ref_min(double a, double b) { return (b < a) ? b : a; }

__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_relaxed_gpu(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned *p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;"
                 : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

__device__ __forceinline__ void red_add_release_gpu(unsigned *p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

// Programmatic dependent launch. A kernel launched with the programmatic
// stream serialization attribute may be scheduled while the kernel before it
// in the stream is still draining. It calls pdl_enter() before touching
// memory: griddepcontrol.wait returns once the previous kernel has completed
// and its writes are visible (so every kernel of such a chain orders after all
// earlier ones), and launch_dependents lets the next kernel's blocks be
// scheduled in turn. In a kernel launched without the attribute both are
// no-ops.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Sum over a warp in a fixed butterfly order; every lane gets the total.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum of one value per thread. All threads must call it;
// every thread receives the total. `scratch` holds >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double *scratch) {
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();  // scratch may still be read by a previous call
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    double t = (threadIdx.x < nw) ? scratch[threadIdx.x] : 0.0;
    if (wid == 0) {
        t = warp_sum(t);
        if (lane == 0) scratch[32] = t;
    }
    __syncthreads();
    return scratch[32];
}

// Deterministic block sum of K values per thread; each value is summed with
// the same tree whatever K is. scratch holds >= 33*K doubles.
template <int K>
__device__ __forceinline__ void block_sum_k(double (&v)[K], double *scratch) {
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) scratch[k * 33 + wid] = v[k];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double t = (lane < nw) ? scratch[k * 33 + lane] : 0.0;
            t = warp_sum(t);
            if (lane == 0) scratch[k * 33 + 32] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = scratch[k * 33 + 32];
}

// Sum of `count` partials (stride 1) read with L1 bypass, in a fixed order
// (thread t takes t, t+blockDim, ...; then block_sum). Every thread gets it.
__device__ __forceinline__ double sum_partials(const double *part, int count, double *scratch) {
    double s = 0.0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) s += __ldcg(part + i);
    return block_sum(s, scratch);
}

// "Last block done" ticket: after each block has stored its partial, the
// block that takes the final ticket sees every partial. Returns true in that
// block (on all its threads) and re-arms the counter for the next launch.
__device__ __forceinline__ bool last_block_done(unsigned *counter) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned ticket = atomicAdd(counter, 1u);
        is_last = (ticket == gridDim.x - 1);
        if (is_last) *counter = 0u;
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

// Status codes written by kernels into a device status word.
constexpr int kStatusOk = 0;
constexpr int kStatusTimeout = -5;   // == KTG_ERR_TIMEOUT
constexpr int kStatusCapacity = -6;  // == KTG_ERR_RANGE

// Grid-wide barrier for cooperative launches, with a deadline. Counter and
// generation live in global memory. Returns false (in every thread of the
// block) when the deadline passed or another block already reported an
// error; the caller must then leave the kernel.
__device__ __forceinline__ bool grid_barrier(unsigned *count, unsigned *gen, int *status,
                                             uint64_t deadline_ns) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const unsigned my_gen = ld_acquire_gpu(gen);
        __threadfence();
        const unsigned arrived = atom_add_acq_rel_gpu(count, 1u);
        if (arrived == gridDim.x - 1) {
            *count = 0u;
            __threadfence();
            red_add_release_gpu(gen, 1u);
        } else {
            uint32_t spins = 0;
            while (ld_acquire_gpu(gen) == my_gen) {
                if ((++spins & 63u) == 0u) {
                    if (ld_relaxed_gpu(status) != kStatusOk || global_timer_ns() > deadline_ns) {
                        atomicCAS(status, kStatusOk, kStatusTimeout);
                        ok = 0;
                        break;
                    }
                }
                __nanosleep(20);
            }
        }
        __threadfence();
        if (ok && ld_relaxed_gpu(status) != kStatusOk) ok = 0;
    }
    __syncthreads();
    return ok != 0;
}

// Grid barrier for the persistent solvers, with grid_barrier's contract but
// fewer round trips to L2 on the critical path: the generation a block waits
// on is kept in a register of thread 0 (read once by grid_sync_init, before
// the first arrival, when every block sees the same value), arriving is one
// acq_rel atomic (its release half publishes the block's writes, ordered
// before it by __syncthreads) and waiting is one acquire load per poll (its
// acquire half orders the block's later reads). Other blocks' errors are
// seen while polling; a block that passes a barrier another block gave up
// on stops at its next one.
struct GridSync {
    unsigned *count;
    unsigned *gen;
    int *status;
    unsigned open_gen;  // meaningful in thread 0 only
};

__device__ __forceinline__ GridSync grid_sync_init(unsigned *count, unsigned *gen, int *status) {
    GridSync g{count, gen, status, 0u};
    if (threadIdx.x == 0) g.open_gen = ld_acquire_gpu(gen);
    return g;
}

__device__ __forceinline__ bool grid_sync(GridSync &g, uint64_t deadline_ns) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        const unsigned arrived = atom_add_acq_rel_gpu(g.count, 1u);
        if (arrived == gridDim.x - 1) {
            *g.count = 0u;
            red_add_release_gpu(g.gen, 1u);
        } else {
            uint32_t spins = 0;
            while (ld_acquire_gpu(g.gen) == g.open_gen) {
                if ((++spins & 63u) == 0u) {
                    if (ld_relaxed_gpu(g.status) != kStatusOk || global_timer_ns() > deadline_ns) {
                        atomicCAS(g.status, kStatusOk, kStatusTimeout);
                        good = 0;
                        break;
                    }
                }
                __nanosleep(20);
            }
        }
        g.open_gen += 1u;
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

}  // namespace ktg
