// Batched Jacobi-PCG over many independent systems (sm_100a).
//
// The solves of solveBothAxes (globalPlacer/simpl/simpl_lss.cc:203-290) for
// many netlists at once -- x and y of each, of uneven sizes -- in one
// persistent launch of thread-block clusters:
//   * one cluster (2-16 CTAs on as many SMs) solves one system at a time; its
//     CTAs split the rows, meet at hardware cluster barriers, and combine
//     their dot-product partials through distributed shared memory in a
//     fixed order (deterministic, identical in every CTA);
//   * clusters take systems from an atomic work queue ordered largest first,
//     so uneven sizes balance without any grid-wide synchronisation;
//   * FP64 Jacobi-PCG (the reference's method), or FP32 Jacobi-PCG inside FP64
//     iterative refinement (true FP64 residual as the convergence test);
//   * per system the device records iterations, the final residual and the
//     solve latency (%globaltimer from dequeue to done).
// The launch only enqueues work, so the whole batch solve is captured once
// in a CUDA graph and replayed.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <functional>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "ktg_common.cuh"
#include "ktg_context.h"
#include "ktg_spmv.cuh"
#include "ktplace_b200.h"

namespace cg = cooperative_groups;

namespace ktg {
namespace {

struct SysDesc {
    int64_t row_base;  // first row in the concatenated vectors
    int64_t nnz_base;  // first entry in col/val
    int32_t n;
    int32_t pad;
};

struct BatchArgs {
    const SysDesc *sys;
    const int32_t *order;  // solve order (largest first)
    int32_t num_sys;
    const int32_t *rp;     // system k's row_ptr (local offsets) at row_base + k
    const int32_t *col;
    const double *val;
    const float *val32;
    const double *diag;
    const double *rhs;
    double *x;
    double *r;
    double *z;
    double *p;
    double *ap;
    float *d32;
    float *ri32;
    float *z32;
    float *p32;
    float *ap32;
    unsigned *queue;
    ktg_batch_result *results;
    double tol;
    double inner_tol;
    int64_t max_iter;
    int32_t max_outer;
    int32_t mixed;
    uint64_t total_timeout_ns;
};

// Cluster-wide deterministic sum of K values per thread. Partials are double
// buffered in shared memory so one cluster barrier per reduction suffices.
template <int K>
__device__ __forceinline__ void cluster_sum(double (&v)[K], double *part, int &buf,
                                            double *scratch, cg::cluster_group &cl) {
    block_sum_k<K>(v, scratch);
    double *mine = part + buf * 4;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) mine[k] = v[k];
    }
    cl.sync();
    const unsigned nb = cl.num_blocks();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double t = 0.0;
        for (unsigned q = 0; q < nb; ++q) t += *cl.map_shared_rank(mine + k, q);
        v[k] = t;
    }
    buf ^= 1;
}

template <typename T, typename V>
__device__ __forceinline__ T row_dot(const int32_t *rp, const int32_t *col, const V *val,
                                     const T *in, int32_t i, T acc) {
    int32_t e = rp[i];
    const int32_t e1 = rp[i + 1];
    for (; e + 4 <= e1; e += 4) {
        const int32_t c0 = __ldg(col + e), c1 = __ldg(col + e + 1);
        const int32_t c2 = __ldg(col + e + 2), c3 = __ldg(col + e + 3);
        const T g0 = __ldcg(in + c0), g1 = __ldcg(in + c1);
        const T g2 = __ldcg(in + c2), g3 = __ldcg(in + c3);
        acc += static_cast<T>(__ldg(val + e)) * g0;
        acc += static_cast<T>(__ldg(val + e + 1)) * g1;
        acc += static_cast<T>(__ldg(val + e + 2)) * g2;
        acc += static_cast<T>(__ldg(val + e + 3)) * g3;
    }
    for (; e < e1; ++e) acc += static_cast<T>(__ldg(val + e)) * __ldcg(in + __ldg(col + e));
    return acc;
}

__global__ void __launch_bounds__(1024) k_batch_pcg(BatchArgs A) {
    cg::cluster_group cl = cg::this_cluster();
    __shared__ double scratch[33 * 4];
    __shared__ double part[2 * 4];
    __shared__ __align__(16) double tilebuf[32 * kTileChunk];  // warp tiles, <= 32 warps
    __shared__ int32_t wb[32 + 1];
    __shared__ int s_job;
    __shared__ int s_stop;
    int buf = 0;
    const unsigned rank = cl.block_rank();
    const unsigned nb = cl.num_blocks();
    const uint64_t deadline = global_timer_ns() + A.total_timeout_ns;
    cl.sync();  // every CTA of the cluster is running before DSMEM is touched

    for (;;) {
        if (rank == 0 && threadIdx.x == 0) {
            s_job = static_cast<int>(atomicAdd(A.queue, 1u));
            s_stop = global_timer_ns() > deadline ? 1 : 0;
        }
        cl.sync();
        const int job = *cl.map_shared_rank(&s_job, 0);
        const bool late = *cl.map_shared_rank(&s_stop, 0) != 0;
        if (job >= A.num_sys) break;
        const int sid = A.order[job];
        const SysDesc S = A.sys[sid];
        const uint64_t t0 = global_timer_ns();
        const int32_t n = S.n;
        const int32_t a = static_cast<int32_t>((static_cast<int64_t>(n) * rank) / nb);
        const int32_t b = static_cast<int32_t>((static_cast<int64_t>(n) * (rank + 1)) / nb);
        const int32_t *rp = A.rp + S.row_base + sid;
        const int32_t *col = A.col + S.nnz_base;
        const double *val = A.val + S.nnz_base;
        const float *val32 = A.val32 + S.nnz_base;
        const double *dg = A.diag + S.row_base;
        const double *rhs = A.rhs + S.row_base;
        double *x = A.x + S.row_base;
        double *r = A.r + S.row_base;

        // per-warp row ranges of the warp tiles, balanced by nonzeros
        warp_row_bounds(b - a, wb, [&](int32_t l) {
            return int64_t(__ldg(rp + a + l)) - __ldg(rp + a) + int64_t(kRowCost) * l;
        });

        ktg_batch_result res;
        res.iters = 0;
        res.outer = 0;
        res.status = late ? KTG_ERR_TIMEOUT : KTG_OK;
        double resid = 0.0;

        if (!A.mixed) {
            double *z = A.z + S.row_base;
            double *p = A.p + S.row_base;
            double *ap = A.ap + S.row_base;
            double v[3] = {0.0, 0.0, 0.0};  // bb, rz, rr
            for (int32_t i = a + threadIdx.x; i < b; i += blockDim.x) {
                const double s = row_dot<double, double>(rp, col, val, x, i, dg[i] * x[i]);
                const double bi = rhs[i];
                const double ri = bi - s;
                const double zi = ri / dg[i];
                r[i] = ri;
                z[i] = zi;
                __stcg(p + i, zi);
                v[0] += bi * bi;
                v[1] += ri * zi;
                v[2] += ri * ri;
            }
            cluster_sum<3>(v, part, buf, scratch, cl);
            const double bnorm = sqrt(v[0]);
            bool active = bnorm > 0.0 && !late;
            double rho = v[1];
            resid = bnorm > 0.0 ? sqrt(v[2]) / bnorm : 0.0;
            int64_t it = 0;
            for (;;) {
                if (!(active && resid > A.tol && it < A.max_iter)) break;
                if (rank == 0 && threadIdx.x == 0) s_stop = global_timer_ns() > deadline ? 1 : 0;
                double w[1] = {0.0};
                double pcur = 0.0;
                warp_tile_spmv<double>(
                    a, INT32_MAX, b - a, kAllAxes, wb, tilebuf,
                    [&](int, const int32_t *&trp, const int32_t *&tcol, const double *&tval,
                        const double *&tin) {
                        trp = rp;
                        tcol = col;
                        tval = val;
                        tin = p;
                    },
                    [&](int32_t, int, int32_t i) {
                        pcur = __ldcg(p + i);
                        return dg[i] * pcur;
                    },
                    [&](int32_t, int, int32_t i, double s) {
                        ap[i] = s;
                        w[0] += pcur * s;
                    });
                cluster_sum<1>(w, part, buf, scratch, cl);
                if (*cl.map_shared_rank(&s_stop, 0)) {
                    res.status = KTG_ERR_TIMEOUT;
                    break;
                }
                const bool ok = w[0] > 0.0;
                const double alpha = ok ? rho / w[0] : 0.0;
                double u[2] = {0.0, 0.0};  // rr, rz
                if (ok) {
                    for (int32_t i = a + threadIdx.x; i < b; i += blockDim.x) {
                        x[i] += alpha * __ldcg(p + i);
                        const double ri = r[i] - alpha * ap[i];
                        const double zi = ri / dg[i];
                        r[i] = ri;
                        z[i] = zi;
                        u[0] += ri * ri;
                        u[1] += ri * zi;
                    }
                }
                cluster_sum<2>(u, part, buf, scratch, cl);
                ++it;
                if (!ok) {
                    active = false;
                    continue;
                }
                resid = sqrt(u[0]) / bnorm;
                if (!(u[1] > 0.0)) {
                    active = false;
                    continue;
                }
                const double beta = u[1] / rho;
                rho = u[1];
                for (int32_t i = a + threadIdx.x; i < b; i += blockDim.x)
                    __stcg(p + i, z[i] + beta * __ldcg(p + i));
                cl.sync();
            }
            res.iters = it;
        } else {
            float *d = A.d32 + S.row_base;
            float *ri = A.ri32 + S.row_base;
            float *z = A.z32 + S.row_base;
            float *p = A.p32 + S.row_base;
            float *ap = A.ap32 + S.row_base;
            double bnorm = 0.0, prev = 0.0;
            int64_t inner = 0;
            int32_t outer = 0;
            for (int round = 0;; ++round) {
                double v[2] = {0.0, 0.0};  // rr, bb
                for (int32_t i = a + threadIdx.x; i < b; i += blockDim.x) {
                    const double s = row_dot<double, double>(rp, col, val, x, i, dg[i] * __ldcg(x + i));
                    const double bi = rhs[i];
                    const double rr = bi - s;
                    r[i] = rr;
                    v[0] += rr * rr;
                    v[1] += bi * bi;
                }
                cluster_sum<2>(v, part, buf, scratch, cl);
                if (round == 0) bnorm = sqrt(v[1]);
                const double rnorm = sqrt(v[0]);
                prev = resid;
                resid = bnorm > 0.0 ? rnorm / bnorm : 0.0;
                const bool stalled = round > 0 && !(resid < 0.5 * prev);
                if (!(bnorm > 0.0) || late || resid <= A.tol || outer >= A.max_outer ||
                    inner >= A.max_iter || stalled) {
                    if (stalled && resid > A.tol) res.status = 1;  // stalled: caller may retry in FP64
                    break;
                }
                double q[2] = {0.0, 0.0};  // rz, rr (inner)
                for (int32_t i = a + threadIdx.x; i < b; i += blockDim.x) {
                    const float rf = static_cast<float>(r[i]);
                    const float zf = rf / static_cast<float>(dg[i]);
                    ri[i] = rf;
                    d[i] = 0.0f;
                    z[i] = zf;
                    __stcg(p + i, zf);
                    q[0] += static_cast<double>(rf) * zf;
                    q[1] += static_cast<double>(rf) * rf;
                }
                cluster_sum<2>(q, part, buf, scratch, cl);
                double rho = q[0];
                double iresid = sqrt(q[1]);
                const double target = A.inner_tol * rnorm;
                bool live = rho > 0.0;
                while (live && iresid > target && inner < A.max_iter) {
                    double w[1] = {0.0};
                    float pcur = 0.0f;
                    warp_tile_spmv<float>(
                        a, INT32_MAX, b - a, kAllAxes, wb, reinterpret_cast<float *>(tilebuf),
                        [&](int, const int32_t *&trp, const int32_t *&tcol, const float *&tval,
                            const float *&tin) {
                            trp = rp;
                            tcol = col;
                            tval = val32;
                            tin = p;
                        },
                        [&](int32_t, int, int32_t i) {
                            pcur = __ldcg(p + i);
                            return static_cast<float>(dg[i]) * pcur;
                        },
                        [&](int32_t, int, int32_t i, float s) {
                            ap[i] = s;
                            w[0] += static_cast<double>(pcur) * s;
                        });
                    cluster_sum<1>(w, part, buf, scratch, cl);
                    ++inner;
                    if (!(w[0] > 0.0)) break;
                    const float alpha = static_cast<float>(rho / w[0]);
                    double u[2] = {0.0, 0.0};
                    for (int32_t i = a + threadIdx.x; i < b; i += blockDim.x) {
                        d[i] += alpha * __ldcg(p + i);
                        const float rr = ri[i] - alpha * ap[i];
                        const float zz = rr / static_cast<float>(dg[i]);
                        ri[i] = rr;
                        z[i] = zz;
                        u[0] += static_cast<double>(rr) * rr;
                        u[1] += static_cast<double>(rr) * zz;
                    }
                    cluster_sum<2>(u, part, buf, scratch, cl);
                    iresid = sqrt(u[0]);
                    if (!(u[1] > 0.0)) break;
                    const float beta = static_cast<float>(u[1] / rho);
                    rho = u[1];
                    for (int32_t i = a + threadIdx.x; i < b; i += blockDim.x)
                        __stcg(p + i, z[i] + beta * __ldcg(p + i));
                    cl.sync();
                }
                for (int32_t i = a + threadIdx.x; i < b; i += blockDim.x) x[i] += d[i];
                ++outer;
                cl.sync();
            }
            res.iters = inner;
            res.outer = outer;
        }
        if (rank == 0 && threadIdx.x == 0) {
            res.resid = resid;
            res.latency_ns = static_cast<int64_t>(global_timer_ns() - t0);
            A.results[sid] = res;
        }
        cl.sync();  // the job word may be rewritten only after every CTA read it
    }
    cl.sync();  // no CTA leaves while another may still read its shared memory
}

}  // namespace
}  // namespace ktg

struct ktg_batch {
    int device = 0;
    int num_sms = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    int64_t launches = 0;       // kernels launched by solves (graph replays included)
    int graph_kernels = 0;      // kernels in the captured graph
    // host mirror of the descriptors
    std::vector<ktg::SysDesc> sys;
    std::vector<int64_t> cost;
    int64_t rows = 0, nnz = 0;     // used
    int64_t cap_rows = 0, cap_nnz = 0, cap_sys = 0, cap_rp = 0;
    // device arrays
    ktg::SysDesc *d_sys = nullptr;
    int32_t *d_order = nullptr;
    int32_t *rp = nullptr;  // rows + num_sys entries
    int32_t *col = nullptr;
    double *val = nullptr;
    float *val32 = nullptr;
    double *diag = nullptr, *rhs = nullptr, *x = nullptr, *x0 = nullptr;
    double *r = nullptr, *z = nullptr, *p = nullptr, *ap = nullptr;
    float *d32 = nullptr, *ri32 = nullptr, *z32 = nullptr, *p32 = nullptr, *ap32 = nullptr;
    unsigned *queue = nullptr;
    ktg_batch_result *results = nullptr;
    bool dirty = true;  // descriptors / order need upload
    // launch shape
    int cluster = 8;
    int threads = 512;
    // size classes: systems of at least split_rows rows (0: none) are solved
    // by a second, concurrent launch of split_clusters clusters of
    // split_cluster CTAs of split_threads threads, with their own queue
    int64_t split_rows = 0;
    int split_cluster = 16, split_threads = 1024, split_clusters = 1;
    int num_large = 0;           // systems in the large class (first in d_order)
    unsigned *queue2 = nullptr;  // the large class's work queue
    int64_t order_split_rows = -1;  // split the uploaded order was built for
    int num_queued = 0;             // systems the cluster launches take (in d_order)
    // whole-GPU path: pairs of consecutive systems of equal size >=
    // offload_rows (the x and y systems of one netlist) are solved one pair
    // after another by an internal context (aggregation-preconditioned mixed
    // solve, or the FP64 solve), before the cluster launches take the rest
    int64_t offload_rows = 0;
    int offload_precond = 2, offload_coarse = 0;
    int64_t order_offload_rows = -1;
    std::vector<int32_t> off_first;  // first system of each offloaded pair
    ktg_ctx *octx = nullptr;
    int64_t octx_launches = 0;
    ktg_mixed_info *d_minfo = nullptr;
    ktg_solve_info *d_sinfo = nullptr;
    unsigned long long *d_stamp = nullptr;
    // graph cache
    cudaGraphExec_t graph = nullptr;
    double g_tol = -1, g_inner = -1;
    int64_t g_max_iter = -1;
    int g_mixed = -1, g_cluster = -1, g_threads = -1;
    int64_t g_split_rows = -1;
    int g_split_cluster = -1, g_split_threads = -1, g_split_clusters = -1;
};

namespace {

int berr(ktg_batch *b, int code, const std::string &m) {
    if (b) b->err = m;
    return code;
}

#define KTG_BCUDA(b, call)                                                          \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess)                                                      \
            return berr((b), KTG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
int grow(ktg_batch *b, T **ptr, int64_t used, int64_t cap) {
    T *np = nullptr;
    KTG_BCUDA(b, cudaMalloc(reinterpret_cast<void **>(&np), sizeof(T) * std::max<int64_t>(cap, 1)));
    if (*ptr && used > 0)
        KTG_BCUDA(b, cudaMemcpyAsync(np, *ptr, sizeof(T) * used, cudaMemcpyDeviceToDevice, b->stream));
    KTG_BCUDA(b, cudaStreamSynchronize(b->stream));
    if (*ptr) cudaFree(*ptr);
    *ptr = np;
    return KTG_OK;
}

// Room for `rows` vector rows, `nnz` entries and `nsys` systems in total.
int reserve(ktg_batch *b, int64_t rows, int64_t nnz, int64_t nsys) {
    int rc;
    if (rows > b->cap_rows) {
        const int64_t cap = std::max(rows, 2 * b->cap_rows);
        const int64_t used = b->rows;
        if ((rc = grow(b, &b->diag, used, cap)) || (rc = grow(b, &b->rhs, used, cap)) ||
            (rc = grow(b, &b->x, used, cap)) || (rc = grow(b, &b->x0, used, cap)) ||
            (rc = grow(b, &b->r, 0, cap)) || (rc = grow(b, &b->z, 0, cap)) ||
            (rc = grow(b, &b->p, 0, cap)) || (rc = grow(b, &b->ap, 0, cap)) ||
            (rc = grow(b, &b->d32, 0, cap)) || (rc = grow(b, &b->ri32, 0, cap)) ||
            (rc = grow(b, &b->z32, 0, cap)) || (rc = grow(b, &b->p32, 0, cap)) ||
            (rc = grow(b, &b->ap32, 0, cap)))
            return rc;
        b->cap_rows = cap;
    }
    if (rows + nsys > b->cap_rp) {
        const int64_t cap = std::max(rows + nsys, 2 * b->cap_rp);
        if ((rc = grow(b, &b->rp, b->rows + static_cast<int64_t>(b->sys.size()), cap))) return rc;
        b->cap_rp = cap;
    }
    if (nsys > b->cap_sys) {
        const int64_t cap = std::max<int64_t>(nsys, 2 * b->cap_sys);
        if ((rc = grow(b, &b->d_sys, 0, cap)) || (rc = grow(b, &b->d_order, 0, cap)) ||
            (rc = grow(b, &b->results, static_cast<int64_t>(b->sys.size()), cap)))
            return rc;
        b->cap_sys = cap;
    }
    if (nnz > b->cap_nnz) {
        const int64_t cap = std::max(nnz, 2 * b->cap_nnz);
        if ((rc = grow(b, &b->col, b->nnz, cap)) || (rc = grow(b, &b->val, b->nnz, cap)) ||
            (rc = grow(b, &b->val32, b->nnz, cap)))
            return rc;
        b->cap_nnz = cap;
    }
    return KTG_OK;
}

__global__ void k_batch_f32(const double *a, float *b, int64_t n) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        b[i] = static_cast<float>(a[i]);
}

__global__ void k_stamp(unsigned long long *t) { *t = ktg::global_timer_ns(); }

// Results of an offloaded pair (systems sx, sy) from its solve's info: the
// mixed solve's inner iterations, rounds and final true residuals (the FP64
// pass's when it ran), or the FP64 solve's iterations and residuals; status
// the solve's error, else 0 when the residual meets tol and 1 when not.
__global__ void k_offload_results(const ktg_mixed_info *mi, const ktg_solve_info *si, int mixed,
                                  double tol, int32_t sx, int32_t sy,
                                  const unsigned long long *t0, ktg_batch_result *res) {
    const int64_t lat = static_cast<int64_t>(ktg::global_timer_ns() - *t0);
    for (int a = 0; a < 2; ++a) {
        ktg_batch_result r;
        if (mixed) {
            r.iters = a ? mi->inner_y : mi->inner_x;
            r.outer = a ? mi->outer_y : mi->outer_x;
            r.resid = a ? mi->resid_y : mi->resid_x;
            r.status = mi->status != 0 ? mi->status : (r.resid <= tol ? 0 : 1);
        } else {
            r.iters = a ? si->iters_y : si->iters_x;
            r.outer = 0;
            r.resid = a ? si->resid_y : si->resid_x;
            r.status = si->status != 0 ? si->status : (r.resid <= tol ? 0 : 1);
        }
        r.latency_ns = lat;
        res[a ? sy : sx] = r;
    }
}

}  // namespace

// Systems that leave the queues for the whole GPU at the current offload
// threshold: consecutive systems of equal size (an x/y pair) of at least
// offload_rows rows, paired from the front.
static std::vector<char> offloaded(const ktg_batch *b, std::vector<int32_t> *first = nullptr) {
    const int32_t ns = static_cast<int32_t>(b->sys.size());
    std::vector<char> off(ns, 0);
    if (first) first->clear();
    if (b->offload_rows > 0) {
        for (int32_t k = 0; k + 1 < ns;) {
            if (b->sys[k].n >= b->offload_rows && b->sys[k + 1].n == b->sys[k].n) {
                if (first) first->push_back(k);
                off[k] = off[k + 1] = 1;
                k += 2;
            } else {
                ++k;
            }
        }
    }
    return off;
}

extern "C" {

int ktg_batch_create(int device, ktg_batch **out) {
    if (!out) return KTG_ERR_ARG;
    *out = nullptr;
    ktg_batch *b = new (std::nothrow) ktg_batch();
    if (!b) return KTG_ERR_NOMEM;
    b->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&b->queue, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&b->queue2, sizeof(unsigned)) != cudaSuccess) {
        ktg_batch_destroy(b);
        return KTG_ERR_CUDA;
    }
    b->stream = b->own_stream;
    *out = b;
    return KTG_OK;
}

void ktg_batch_destroy(ktg_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    void *ptrs[] = {b->d_sys, b->d_order, b->rp, b->col, b->val, b->val32, b->diag, b->rhs,
                    b->x, b->x0, b->r, b->z, b->p, b->ap, b->d32, b->ri32, b->z32, b->p32,
                    b->ap32, b->queue, b->queue2, b->results, b->d_minfo, b->d_sinfo,
                    b->d_stamp};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (b->octx) ktg_destroy(b->octx);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    delete b;
}

const char *ktg_batch_last_error(const ktg_batch *b) { return b ? b->err.c_str() : "null batch"; }

int ktg_batch_set_stream(ktg_batch *b, void *stream) {
    if (!b) return KTG_ERR_ARG;
    b->stream = stream ? static_cast<cudaStream_t>(stream) : b->own_stream;
    return KTG_OK;
}

int64_t ktg_batch_size(const ktg_batch *b) { return b ? static_cast<int64_t>(b->sys.size()) : 0; }

int ktg_batch_add_system(ktg_batch *b, int64_t n, const int64_t *row_ptr, const int32_t *col,
                         const double *val, const double *diag, const double *rhs,
                         const double *x0, int64_t *id) {
    if (!b || n < 0 || !row_ptr || (n > 0 && (!diag || !rhs || !x0))) return KTG_ERR_ARG;
    const int64_t m = row_ptr[n];
    if (m < 0 || (m > 0 && (!col || !val))) return KTG_ERR_ARG;
    if (n > 0x3fffffffll || m > 0x7fffffffll || b->rows + n > 0x7fffffffll ||
        b->nnz + m > 0x7fffffffll)
        return berr(b, KTG_ERR_RANGE, "batch exceeds 32-bit indices");
    std::vector<int32_t> rp(n + 1);
    for (int64_t i = 0; i <= n; ++i) {
        if (row_ptr[i] < 0 || (i > 0 && row_ptr[i] < row_ptr[i - 1]))
            return berr(b, KTG_ERR_ARG, "row_ptr not monotone");
        rp[i] = static_cast<int32_t>(row_ptr[i]);
    }
    for (int64_t e = 0; e < m; ++e)
        if (col[e] < 0 || col[e] >= n) return berr(b, KTG_ERR_ARG, "col out of range");
    if (cudaSetDevice(b->device) != cudaSuccess) return KTG_ERR_CUDA;
    const int64_t nsys = static_cast<int64_t>(b->sys.size()) + 1;
    int rc = reserve(b, b->rows + n, b->nnz + m, nsys);
    if (rc) return rc;
    const int64_t base = b->rows, ebase = b->nnz, k = nsys - 1;
    KTG_BCUDA(b, cudaMemcpyAsync(b->rp + base + k, rp.data(), sizeof(int32_t) * (n + 1),
                                 cudaMemcpyHostToDevice, b->stream));
    if (m) {
        KTG_BCUDA(b, cudaMemcpyAsync(b->col + ebase, col, sizeof(int32_t) * m, cudaMemcpyHostToDevice, b->stream));
        KTG_BCUDA(b, cudaMemcpyAsync(b->val + ebase, val, sizeof(double) * m, cudaMemcpyHostToDevice, b->stream));
    }
    if (n) {
        KTG_BCUDA(b, cudaMemcpyAsync(b->diag + base, diag, sizeof(double) * n, cudaMemcpyHostToDevice, b->stream));
        KTG_BCUDA(b, cudaMemcpyAsync(b->rhs + base, rhs, sizeof(double) * n, cudaMemcpyHostToDevice, b->stream));
        KTG_BCUDA(b, cudaMemcpyAsync(b->x + base, x0, sizeof(double) * n, cudaMemcpyHostToDevice, b->stream));
        KTG_BCUDA(b, cudaMemcpyAsync(b->x0 + base, x0, sizeof(double) * n, cudaMemcpyHostToDevice, b->stream));
    }
    if (m) {
        k_batch_f32<<<static_cast<int>(std::min<int64_t>((m + 255) / 256, 4096)), 256, 0, b->stream>>>(
            b->val + ebase, b->val32 + ebase, m);
        ++b->launches;
    }
    KTG_BCUDA(b, cudaStreamSynchronize(b->stream));
    b->sys.push_back(ktg::SysDesc{base, ebase, static_cast<int32_t>(n), 0});
    b->cost.push_back(m + n);
    b->rows += n;
    b->nnz += m;
    b->dirty = true;
    if (id) *id = k;
    return KTG_OK;
}

int ktg_batch_add_from_context(ktg_batch *b, ktg_ctx *c, const double *x0, const double *y0,
                               int64_t *first_id) {
    if (!b || !c || !x0 || !y0) return KTG_ERR_ARG;
    if (!c->have_system) return berr(b, KTG_ERR_STATE, "context has no systems");
    int64_t first = -1;
    for (int axis = 0; axis < 2; ++axis) {
        int64_t n = 0, m = 0;
        int rc = ktg_system_info(c, axis, &n, &m);
        if (rc) return berr(b, rc, "ktg_system_info failed");
        std::vector<int64_t> rp(n + 1);
        std::vector<int32_t> col(m);
        std::vector<double> val(m), dg(n), rhs(n);
        if ((rc = ktg_download_system(c, axis, rp.data(), col.data(), val.data(), dg.data(), rhs.data())))
            return berr(b, rc, "ktg_download_system failed");
        int64_t id = -1;
        if ((rc = ktg_batch_add_system(b, n, rp.data(), col.data(), val.data(), dg.data(), rhs.data(),
                                       axis ? y0 : x0, &id)))
            return rc;
        if (axis == 0) first = id;
    }
    if (first_id) *first_id = first;
    return KTG_OK;
}

int ktg_batch_set_shape(ktg_batch *b, int cluster, int threads) {
    if (!b) return KTG_ERR_ARG;
    if (!(cluster == 1 || cluster == 2 || cluster == 4 || cluster == 8 || cluster == 16))
        return berr(b, KTG_ERR_ARG, "cluster must be 1, 2, 4, 8 or 16");
    if (!(threads == 128 || threads == 256 || threads == 512 || threads == 1024))
        return berr(b, KTG_ERR_ARG, "threads must be 128, 256, 512 or 1024");
    b->cluster = cluster;
    b->threads = threads;
    return KTG_OK;
}

int ktg_batch_get_shape(const ktg_batch *b, int *cluster, int *threads) {
    if (!b) return KTG_ERR_ARG;
    if (cluster) *cluster = b->cluster;
    if (threads) *threads = b->threads;
    return KTG_OK;
}

int ktg_batch_set_split(ktg_batch *b, int64_t rows, int cluster, int threads, int clusters) {
    if (!b) return KTG_ERR_ARG;
    if (rows < 0) return berr(b, KTG_ERR_ARG, "negative split rows");
    if (rows > 0) {
        if (!(cluster == 1 || cluster == 2 || cluster == 4 || cluster == 8 || cluster == 16))
            return berr(b, KTG_ERR_ARG, "cluster must be 1, 2, 4, 8 or 16");
        if (!(threads == 128 || threads == 256 || threads == 512 || threads == 1024))
            return berr(b, KTG_ERR_ARG, "threads must be 128, 256, 512 or 1024");
        if (clusters < 1) return berr(b, KTG_ERR_ARG, "clusters must be >= 1");
        b->split_cluster = cluster;
        b->split_threads = threads;
        b->split_clusters = clusters;
    }
    b->split_rows = rows;
    return KTG_OK;
}

int ktg_batch_set_offload(ktg_batch *b, int64_t rows, int precond, int coarse) {
    if (!b) return KTG_ERR_ARG;
    if (rows < 0) return berr(b, KTG_ERR_ARG, "negative offload rows");
    if (precond < 0 || precond > 2) return berr(b, KTG_ERR_ARG, "precond must be 0, 1 or 2");
    if (coarse < 0 || coarse > 2) return berr(b, KTG_ERR_ARG, "coarse must be 0, 1 or 2");
    if (precond == 1) return berr(b, KTG_ERR_ARG, "the learned inverse needs a prepared network");
    b->offload_rows = rows;
    b->offload_precond = precond;
    b->offload_coarse = coarse;
    return KTG_OK;
}

int ktg_batch_get_offload(const ktg_batch *b, int64_t *rows, int *pairs) {
    if (!b) return KTG_ERR_ARG;
    if (rows) *rows = b->offload_rows;
    if (pairs) {
        int k = 0;
        const int32_t ns = static_cast<int32_t>(b->sys.size());
        if (b->offload_rows > 0)
            for (int32_t i = 0; i + 1 < ns;) {
                if (b->sys[i].n >= b->offload_rows && b->sys[i + 1].n == b->sys[i].n) {
                    ++k;
                    i += 2;
                } else {
                    ++i;
                }
            }
        *pairs = k;
    }
    return KTG_OK;
}

int ktg_batch_get_split(const ktg_batch *b, int64_t *rows, int *cluster, int *threads,
                        int *clusters, int *num_large) {
    if (!b) return KTG_ERR_ARG;
    if (rows) *rows = b->split_rows;
    if (cluster) *cluster = b->split_cluster;
    if (threads) *threads = b->split_threads;
    if (clusters) *clusters = b->split_clusters;
    if (num_large) {
        // systems of the queues only: offloaded pairs are in no class
        const std::vector<char> off = offloaded(b);
        int64_t k = 0;
        if (b->split_rows > 0)
            for (size_t i = 0; i < b->sys.size(); ++i) k += !off[i] && b->sys[i].n >= b->split_rows;
        *num_large = static_cast<int>(k);
    }
    return KTG_OK;
}

int ktg_batch_reset_x(ktg_batch *b) {
    if (!b) return KTG_ERR_ARG;
    if (b->rows)
        KTG_BCUDA(b, cudaMemcpyAsync(b->x, b->x0, sizeof(double) * b->rows, cudaMemcpyDeviceToDevice,
                                     b->stream));
    return KTG_OK;
}

// How many clusters of `cluster` CTAs of `threads` threads can be resident
// at once on the whole device.
static int resident_clusters(ktg_batch *b, int cluster, int threads, int *out) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(threads);
    cfg.gridDim = dim3(cluster);
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cluster > 8)
        KTG_BCUDA(b, cudaFuncSetAttribute(ktg::k_batch_pcg,
                                          cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    KTG_BCUDA(b, cudaOccupancyMaxActiveClusters(out, ktg::k_batch_pcg, &cfg));
    if (*out < 1) return berr(b, KTG_ERR_CUDA, "cluster shape cannot be resident");
    return KTG_OK;
}

// One persistent launch over the systems order[first, first + count): `clusters`
// clusters of `cluster` CTAs of `threads` threads draining `queue`.
static int enqueue_class(ktg_batch *b, int first, int count, unsigned *queue, int cluster,
                         int threads, int clusters, double tol, int64_t max_iter, int mixed,
                         double inner_tol, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(std::max(1, std::min(clusters, count)) * cluster);
    ktg::BatchArgs A{b->d_sys, b->d_order + first, count, b->rp, b->col, b->val, b->val32,
                     b->diag, b->rhs, b->x, b->r, b->z, b->p, b->ap, b->d32, b->ri32, b->z32,
                     b->p32, b->ap32, queue, b->results, tol, inner_tol, max_iter, 50, mixed,
                     120000000000ull};
    KTG_BCUDA(b, cudaMemsetAsync(queue, 0, sizeof(unsigned), st));
    KTG_BCUDA(b, cudaLaunchKernelEx(&cfg, ktg::k_batch_pcg, A));
    return KTG_OK;
}

// Enqueues the whole batch solve on `st`. Without a size split it is one
// launch of the batch shape sized to the device. With one, the large class
// runs on a forked stream as its own launch while the small class's grid is
// cut to the SMs the large clusters leave free; the two launches share no
// state besides the solution arrays of disjoint systems, so neither waits on
// the other and the fork is joined back into `st` at the end.
static int batch_enqueue(ktg_batch *b, double tol, int64_t max_iter, int mixed, double inner_tol,
                         cudaStream_t st) {
    const int ns = b->num_queued;
    const int nl = b->num_large;
    int res_small = 0;
    int rc = resident_clusters(b, b->cluster, b->threads, &res_small);
    if (rc) return rc;
    if (nl == 0) {
        rc = enqueue_class(b, 0, ns, b->queue, b->cluster, b->threads, res_small, tol, max_iter,
                           mixed, inner_tol, st);
        b->graph_kernels = 1;
        return rc;
    }
    int res_large = 0;
    if ((rc = resident_clusters(b, b->split_cluster, b->split_threads, &res_large))) return rc;
    const int large_clusters = std::min({b->split_clusters, res_large, nl});
    if (nl == ns) {
        rc = enqueue_class(b, 0, ns, b->queue2, b->split_cluster, b->split_threads, large_clusters,
                           tol, max_iter, mixed, inner_tol, st);
        b->graph_kernels = 1;
        return rc;
    }
    // SMs held by the large class, from its CTAs per SM when the device is full.
    const int sms = std::max(1, b->num_sms);
    const int large_per_sm = std::max(1, res_large * b->split_cluster / sms);
    const int large_sms = (large_clusters * b->split_cluster + large_per_sm - 1) / large_per_sm;
    const int small_per_sm = std::max(1, res_small * b->cluster / sms);
    const int free_sms = std::max(b->cluster, sms - large_sms);
    const int small_clusters = std::max(1, std::min(res_small, free_sms * small_per_sm / b->cluster));
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaStream_t side = nullptr;
    KTG_BCUDA(b, cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    if (cudaEventCreateWithFlags(&join, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking) != cudaSuccess) {
        cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        return berr(b, KTG_ERR_CUDA, "fork stream creation failed");
    }
    if (cudaEventRecord(fork, st) != cudaSuccess || cudaStreamWaitEvent(side, fork, 0) != cudaSuccess)
        rc = berr(b, KTG_ERR_CUDA, "stream fork failed");
    if (!rc)
        rc = enqueue_class(b, 0, nl, b->queue2, b->split_cluster, b->split_threads, large_clusters,
                           tol, max_iter, mixed, inner_tol, side);
    if (!rc)
        rc = enqueue_class(b, nl, ns - nl, b->queue, b->cluster, b->threads, small_clusters, tol,
                           max_iter, mixed, inner_tol, st);
    if (!rc && (cudaEventRecord(join, side) != cudaSuccess ||
                cudaStreamWaitEvent(st, join, 0) != cudaSuccess))
        rc = berr(b, KTG_ERR_CUDA, "stream join failed");
    cudaEventDestroy(fork);
    cudaEventDestroy(join);
    cudaStreamDestroy(side);
    b->graph_kernels = 2;
    return rc;
}

// The offloaded pairs, one after another on the batch's stream, each through
// the internal context: its x and y systems copied in (device to device),
// then the whole-GPU solve on the batch's own solution slices, then the
// pair's results.
static int solve_offloaded(ktg_batch *b, double tol, int64_t max_iter, int precision,
                           double inner_tol) {
    int rc;
    if (!b->octx) {
        if ((rc = ktg_create(b->device, &b->octx))) return berr(b, rc, "internal context");
        if (cudaMalloc(&b->d_minfo, sizeof(ktg_mixed_info)) != cudaSuccess ||
            cudaMalloc(&b->d_sinfo, sizeof(ktg_solve_info)) != cudaSuccess ||
            cudaMalloc(&b->d_stamp, sizeof(unsigned long long)) != cudaSuccess)
            return berr(b, KTG_ERR_NOMEM, "offload buffers");
    }
    ktg_ctx *c = b->octx;
    const int64_t launches0 = c->launches;
    if ((rc = ktg_set_stream(c, b->stream)) || (rc = ktg_set_pointer_mode(c, KTG_PTR_DEVICE)) ||
        (rc = ktg_set_option(c, "precond", b->offload_precond)) ||
        (rc = ktg_set_option(c, "coarse", b->offload_coarse)))
        return berr(b, rc, std::string("internal context: ") + c->err);
    for (int32_t f : b->off_first) {
        const ktg::SysDesc &X = b->sys[f], &Y = b->sys[f + 1];
        k_stamp<<<1, 1, 0, b->stream>>>(b->d_stamp);
        ++b->launches;
        const int64_t mx = b->cost[f] - X.n, my = b->cost[f + 1] - Y.n;
        // room for both axes at once (one growth at most)
        if ((rc = ktg::reserve_system_arrays(c, X.n, std::max(mx, my))) ||
            (rc = ktg::load_system_device(c, 0, X.n, mx, b->rp + X.row_base + f,
                                          b->col + X.nnz_base, b->val + X.nnz_base,
                                          b->diag + X.row_base, b->rhs + X.row_base)) ||
            (rc = ktg::load_system_device(c, 1, Y.n, my, b->rp + Y.row_base + f + 1,
                                          b->col + Y.nnz_base, b->val + Y.nnz_base,
                                          b->diag + Y.row_base, b->rhs + Y.row_base)))
            return berr(b, rc, std::string("offload load: ") + c->err);
        if (!c->have_system) return berr(b, KTG_ERR_STATE, "offload load: pair not complete");
        double *x = b->x + X.row_base, *y = b->x + Y.row_base;
        rc = precision == 1 ? ktg_solve_mixed(c, x, y, tol, inner_tol, max_iter, 50, b->d_minfo,
                                              nullptr, nullptr, 0)
                            : ktg_solve(c, x, y, tol, max_iter, b->d_sinfo, nullptr, nullptr, 0);
        if (rc) return berr(b, rc, std::string("offload solve: ") + c->err);
        k_offload_results<<<1, 1, 0, b->stream>>>(b->d_minfo, b->d_sinfo, precision, tol, f,
                                                        f + 1, b->d_stamp, b->results);
        ++b->launches;
        KTG_BCUDA(b, cudaGetLastError());
    }
    b->launches += c->launches - launches0;
    return KTG_OK;
}

int ktg_batch_solve(ktg_batch *b, double tol, int64_t max_iter, int precision, double inner_tol) {
    if (!b) return KTG_ERR_ARG;
    if (precision != 0 && precision != 1) return berr(b, KTG_ERR_ARG, "precision must be 0 or 1");
    if (precision == 1 && !(inner_tol > 0.0 && inner_tol < 1.0))
        return berr(b, KTG_ERR_ARG, "inner_tol must be in (0, 1)");
    if (max_iter < 0) return berr(b, KTG_ERR_ARG, "negative max_iter");
    if (b->sys.empty()) return KTG_OK;
    if (cudaSetDevice(b->device) != cudaSuccess) return KTG_ERR_CUDA;
    if (b->dirty || b->order_split_rows != b->split_rows ||
        b->order_offload_rows != b->offload_rows) {
        // Offloaded pairs first leave the queues; then largest first within
        // each class, the large class (rows >= split_rows) at the front.
        const int32_t ns = static_cast<int32_t>(b->sys.size());
        const std::vector<char> off = offloaded(b, &b->off_first);
        std::vector<int32_t> order;
        for (int32_t k = 0; k < ns; ++k)
            if (!off[k]) order.push_back(k);
        b->num_queued = static_cast<int>(order.size());
        auto large = [&](int32_t p) { return b->split_rows > 0 && b->sys[p].n >= b->split_rows; };
        std::stable_sort(order.begin(), order.end(), [&](int32_t p, int32_t q) {
            if (large(p) != large(q)) return large(p);
            return b->cost[p] > b->cost[q];
        });
        b->num_large = static_cast<int>(std::count_if(order.begin(), order.end(), large));
        KTG_BCUDA(b, cudaMemcpyAsync(b->d_sys, b->sys.data(), sizeof(ktg::SysDesc) * b->sys.size(),
                                     cudaMemcpyHostToDevice, b->stream));
        if (!order.empty())
            KTG_BCUDA(b, cudaMemcpyAsync(b->d_order, order.data(), sizeof(int32_t) * order.size(),
                                         cudaMemcpyHostToDevice, b->stream));
        KTG_BCUDA(b, cudaStreamSynchronize(b->stream));
        b->dirty = false;
        b->order_split_rows = b->split_rows;
        b->order_offload_rows = b->offload_rows;
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
    }
    if (!b->off_first.empty()) {
        int rc = solve_offloaded(b, tol, max_iter, precision, inner_tol);
        if (rc) return rc;
    }
    if (b->num_queued == 0) return KTG_OK;
    const bool same = b->graph && b->g_tol == tol && b->g_max_iter == max_iter &&
                      b->g_mixed == precision && b->g_inner == inner_tol &&
                      b->g_cluster == b->cluster && b->g_threads == b->threads &&
                      b->g_split_rows == b->split_rows && b->g_split_cluster == b->split_cluster &&
                      b->g_split_threads == b->split_threads &&
                      b->g_split_clusters == b->split_clusters;
    if (!same) {
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        // Capture the whole batch solve once on a private stream.
        cudaStream_t cap;
        KTG_BCUDA(b, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        int rc = KTG_OK;
        if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaStreamDestroy(cap);
            return berr(b, KTG_ERR_CUDA, "stream capture failed to start");
        }
        rc = batch_enqueue(b, tol, max_iter, precision, inner_tol, cap);
        const cudaError_t ec = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ec != cudaSuccess) return berr(b, KTG_ERR_CUDA, "stream capture failed");
        const cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) return berr(b, KTG_ERR_CUDA, "graph instantiation failed");
        b->g_tol = tol;
        b->g_max_iter = max_iter;
        b->g_mixed = precision;
        b->g_inner = inner_tol;
        b->g_cluster = b->cluster;
        b->g_threads = b->threads;
        b->g_split_rows = b->split_rows;
        b->g_split_cluster = b->split_cluster;
        b->g_split_threads = b->split_threads;
        b->g_split_clusters = b->split_clusters;
    }
    KTG_BCUDA(b, cudaGraphLaunch(b->graph, b->stream));
    b->launches += b->graph_kernels;
    return KTG_OK;
}

int ktg_batch_results(ktg_batch *b, ktg_batch_result *out) {
    if (!b || !out) return KTG_ERR_ARG;
    if (b->sys.empty()) return KTG_OK;
    KTG_BCUDA(b, cudaMemcpyAsync(out, b->results, sizeof(ktg_batch_result) * b->sys.size(),
                                 cudaMemcpyDeviceToHost, b->stream));
    KTG_BCUDA(b, cudaStreamSynchronize(b->stream));
    return KTG_OK;
}

int ktg_batch_get_x(ktg_batch *b, int64_t id, double *x) {
    if (!b || !x || id < 0 || id >= static_cast<int64_t>(b->sys.size())) return KTG_ERR_ARG;
    const ktg::SysDesc &s = b->sys[id];
    KTG_BCUDA(b, cudaMemcpyAsync(x, b->x + s.row_base, sizeof(double) * s.n, cudaMemcpyDeviceToHost,
                                 b->stream));
    KTG_BCUDA(b, cudaStreamSynchronize(b->stream));
    return KTG_OK;
}

int64_t ktg_batch_launch_count(const ktg_batch *b) { return b ? b->launches : 0; }

int ktg_batch_autotune(ktg_batch *b, double tol, int precision, double inner_tol,
                       int64_t probe_iter, int *cluster, int *threads, float *best_ms) {
    if (!b || probe_iter <= 0) return KTG_ERR_ARG;
    if (b->sys.empty()) return berr(b, KTG_ERR_STATE, "empty batch");
    static const int kClusters[] = {2, 4, 8, 16};
    static const int kThreads[] = {256, 512, 1024};
    cudaEvent_t e0, e1;
    KTG_BCUDA(b, cudaEventCreate(&e0));
    KTG_BCUDA(b, cudaEventCreate(&e1));
    float best = 1e30f;
    int bc = b->cluster, bt = b->threads;
    int rc = KTG_OK;
    for (int c : kClusters) {
        for (int t : kThreads) {
            if ((rc = ktg_batch_set_shape(b, c, t))) break;
            int resident = 0;
            if (resident_clusters(b, c, t, &resident) != KTG_OK) {
                b->err.clear();
                continue;  // shape not launchable on this device
            }
            float ms = 0.0f;
            for (int rep = 0; rep < 2 && rc == KTG_OK; ++rep) {
                if ((rc = ktg_batch_reset_x(b))) break;
                if (cudaEventRecord(e0, b->stream) != cudaSuccess) rc = KTG_ERR_CUDA;
                if (!rc) rc = ktg_batch_solve(b, tol, probe_iter, precision, inner_tol);
                if (!rc && cudaEventRecord(e1, b->stream) != cudaSuccess) rc = KTG_ERR_CUDA;
                if (!rc && cudaEventSynchronize(e1) != cudaSuccess) rc = KTG_ERR_CUDA;
                if (!rc) cudaEventElapsedTime(&ms, e0, e1);
            }
            if (rc) break;
            if (ms < best) {
                best = ms;
                bc = c;
                bt = t;
            }
        }
        if (rc) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    ktg_batch_set_shape(b, bc, bt);
    if ((rc = ktg_batch_reset_x(b))) return rc;
    if (cluster) *cluster = bc;
    if (threads) *threads = bt;
    if (best_ms) *best_ms = best;
    return KTG_OK;
}

// Times one full solve (from reset x) of the current configuration.
static int time_solve(ktg_batch *b, double tol, int64_t max_iter, int precision, double inner_tol,
                      cudaEvent_t e0, cudaEvent_t e1, float *ms) {
    int rc;
    if ((rc = ktg_batch_reset_x(b))) return rc;
    KTG_BCUDA(b, cudaEventRecord(e0, b->stream));
    if ((rc = ktg_batch_solve(b, tol, max_iter, precision, inner_tol))) return rc;
    KTG_BCUDA(b, cudaEventRecord(e1, b->stream));
    KTG_BCUDA(b, cudaEventSynchronize(e1));
    KTG_BCUDA(b, cudaEventElapsedTime(ms, e0, e1));
    return KTG_OK;
}

int ktg_batch_autotune_split(ktg_batch *b, double tol, int precision, double inner_tol,
                             int64_t max_iter, float *base_ms, float *best_ms) {
    if (!b || max_iter <= 0) return KTG_ERR_ARG;
    if (b->sys.empty()) return berr(b, KTG_ERR_STATE, "empty batch");
    // Thresholds that put the 1, 2, 4, 8 or 16 largest queued systems (ties
    // included) in the large class; offloaded pairs are in no class.
    std::vector<int64_t> sizes;
    const std::vector<char> off = offloaded(b);
    for (size_t i = 0; i < b->sys.size(); ++i)
        if (!off[i]) sizes.push_back(b->sys[i].n);
    if (sizes.empty()) {  // every system is offloaded: nothing to split
        if (base_ms) *base_ms = 0.0f;
        if (best_ms) *best_ms = 0.0f;
        return ktg_batch_set_split(b, 0, 0, 0, 0);
    }
    std::sort(sizes.begin(), sizes.end(), std::greater<int64_t>());
    std::vector<int64_t> cuts;
    for (size_t k : {1, 2, 4, 8, 16}) {
        if (k >= sizes.size()) break;
        const int64_t t = sizes[k - 1];
        if (t > sizes.back() && (cuts.empty() || cuts.back() != t)) cuts.push_back(t);
    }
    static const int kShapes[][2] = {{16, 1024}, {8, 1024}, {16, 512}};
    static const int kCount[] = {1, 2, 4, 8};
    cudaEvent_t e0, e1;
    KTG_BCUDA(b, cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return berr(b, KTG_ERR_CUDA, "event creation failed");
    }
    int rc = ktg_batch_set_split(b, 0, 0, 0, 0);
    float none = 0.0f, ms = 0.0f;
    for (int rep = 0; rep < 2 && !rc; ++rep) rc = time_solve(b, tol, max_iter, precision, inner_tol, e0, e1, &none);
    float best = none;
    int64_t br = 0;
    int bc = b->split_cluster, bt = b->split_threads, bn = b->split_clusters;
    for (int64_t cut : cuts) {
        if (rc) break;
        for (const auto &sh : kShapes) {
            if (rc) break;
            int resident = 0;
            if (resident_clusters(b, sh[0], sh[1], &resident) != KTG_OK) {
                b->err.clear();
                continue;  // shape not launchable on this device
            }
            for (int n : kCount) {
                if (n > resident) break;
                if ((rc = ktg_batch_set_split(b, cut, sh[0], sh[1], n))) break;
                int nl = 0;
                ktg_batch_get_split(b, nullptr, nullptr, nullptr, nullptr, &nl);
                if (n > nl) break;
                float t = 1e30f;
                for (int rep = 0; rep < 2 && !rc; ++rep) {
                    rc = time_solve(b, tol, max_iter, precision, inner_tol, e0, e1, &ms);
                    t = std::min(t, ms);
                }
                if (!rc && t < best) {
                    best = t;
                    br = cut;
                    bc = sh[0];
                    bt = sh[1];
                    bn = n;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if ((rc = ktg_batch_set_split(b, br, bc, bt, bn))) return rc;
    if ((rc = ktg_batch_reset_x(b))) return rc;
    if (base_ms) *base_ms = none;
    if (best_ms) *best_ms = best;
    return KTG_OK;
}

int ktg_batch_autotune_offload(ktg_batch *b, double tol, int precision, double inner_tol,
                               int64_t max_iter, float *base_ms, float *best_ms) {
    if (!b || max_iter <= 0) return KTG_ERR_ARG;
    if (b->sys.empty()) return berr(b, KTG_ERR_STATE, "empty batch");
    std::vector<int64_t> sizes;
    for (const ktg::SysDesc &d : b->sys) sizes.push_back(d.n);
    std::sort(sizes.begin(), sizes.end(), std::greater<int64_t>());
    std::vector<int64_t> cuts;  // the 2, 4, ... 64 largest systems (pairs of them)
    for (size_t k : {2, 4, 8, 16, 24, 32, 48, 64}) {
        if (k > sizes.size()) break;
        const int64_t t = sizes[k - 1];
        if (t > 0 && (cuts.empty() || cuts.back() != t)) cuts.push_back(t);
    }
    cudaEvent_t e0, e1;
    KTG_BCUDA(b, cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return berr(b, KTG_ERR_CUDA, "event creation failed");
    }
    const int64_t split0 = b->split_rows;
    int rc = ktg_batch_set_split(b, 0, 0, 0, 0);
    const int pre = b->offload_precond, co = b->offload_coarse;
    if (!rc) rc = ktg_batch_set_offload(b, 0, pre, co);
    float none = 1e30f, ms = 0.0f;
    for (int rep = 0; rep < 2 && !rc; ++rep) {
        rc = time_solve(b, tol, max_iter, precision, inner_tol, e0, e1, &ms);
        none = std::min(none, ms);
    }
    float best = none;
    int64_t br = 0;
    for (int64_t cut : cuts) {
        if (rc) break;
        if ((rc = ktg_batch_set_offload(b, cut, pre, co))) break;
        int pairs = 0;
        ktg_batch_get_offload(b, nullptr, &pairs);
        if (pairs == 0) continue;
        float t = 1e30f;
        for (int rep = 0; rep < 2 && !rc; ++rep) {
            rc = time_solve(b, tol, max_iter, precision, inner_tol, e0, e1, &ms);
            t = std::min(t, ms);
        }
        if (!rc && t < best) {
            best = t;
            br = cut;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if ((rc = ktg_batch_set_offload(b, br, pre, co))) return rc;
    b->split_rows = split0;
    if ((rc = ktg_batch_reset_x(b))) return rc;
    if (base_ms) *base_ms = none;
    if (best_ms) *best_ms = best;
    return KTG_OK;
}

}  // extern "C"
