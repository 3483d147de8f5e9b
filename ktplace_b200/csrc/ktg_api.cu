// C ABI of ktplace_b200: context management, netlist/grid upload, and the
// entry points declared in include/ktplace_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "ktg_agg.h"
#include "ktg_context.h"
#include "ktplace_b200.h"

namespace ktg {

int set_error(ktg_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_check(ktg_ctx *ctx, cudaError_t e, const char *what) {
    return set_error(ctx, KTG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace ktg

namespace {

using ktg::set_error;

template <typename T>
int dev_alloc(ktg_ctx *c, T **p, int64_t count) {
    if (*p) {
        cudaFree(*p);
        *p = nullptr;
    }
    if (count <= 0) count = 1;
    const cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * count);
    if (e != cudaSuccess) return ktg::cuda_check(c, e, "cudaMalloc");
    return KTG_OK;
}

template <typename T>
void dev_free(T *&p) {
    if (p) cudaFree(p);
    p = nullptr;
}

template <typename T>
int upload(ktg_ctx *c, T *dst, const T *src, int64_t count) {
    if (count <= 0) return KTG_OK;
    KTG_CUDA(c, cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyHostToDevice, c->stream));
    return KTG_OK;
}

int sync(ktg_ctx *c) {
    KTG_CUDA(c, cudaStreamSynchronize(c->stream));
    return KTG_OK;
}

// Reads the device status word; returns its KTG code (0 when fine).
int device_status(ktg_ctx *c) {
    KTG_CUDA(c, cudaMemcpyAsync(c->h_status, c->status, sizeof(int), cudaMemcpyDeviceToHost,
                                c->stream));
    KTG_CUDA(c, cudaStreamSynchronize(c->stream));
    return *c->h_status;
}

int set_device(ktg_ctx *c) {
    KTG_CUDA(c, cudaSetDevice(c->device));
    return KTG_OK;
}

void free_netlist(ktg_ctx *c) {
    dev_free(c->var_of_vertex);
    dev_free(c->fixed_x);
    dev_free(c->fixed_y);
    dev_free(c->net_start);
    dev_free(c->pin_cell);
    dev_free(c->pin_var);
    dev_free(c->off_x);
    dev_free(c->off_y);
    dev_free(c->net_base);
    dev_free(c->net_weight);
    dev_free(c->net_mov);
    dev_free(c->pin_start);
    dev_free(c->pin_ref);
    dev_free(c->width);
    dev_free(c->height);
    dev_free(c->area);
    dev_free(c->row_cnt);
    dev_free(c->heavy_rows);
    dev_free(c->block_sum);
    c->have_netlist = false;
}

void free_systems(ktg_ctx *c) {
    for (auto &s : c->sys) {
        dev_free(s.row_ptr);
        dev_free(s.col);
        dev_free(s.val);
        dev_free(s.diag);
        dev_free(s.rhs);
        dev_free(s.lo);
        dev_free(s.hi);
        dev_free(s.r);
        dev_free(s.z);
        dev_free(s.p);
        dev_free(s.ap);
        dev_free(s.s);
        dev_free(s.val32);
        dev_free(s.d32);
        dev_free(s.r32);
        dev_free(s.z32);
        dev_free(s.p32);
        dev_free(s.ap32);
        dev_free(s.s32);
        dev_free(s.rs32);
    }
    dev_free(c->x);
    dev_free(c->y);
    dev_free(c->ax);
    dev_free(c->ay);
    c->sys_cap_n = 0;
    c->sys_cap_nnz = 0;
    c->stage_cap = 0;
    c->have_system = false;
    c->axis_valid[0] = c->axis_valid[1] = false;
}

// Makes room for systems of `rows` rows and `nnz` entries per axis and for
// per-net bound pins of the current netlist.
// A larger array that keeps the first `keep` elements of the old one (the
// copy is stream-ordered; cudaFree waits for it).
template <typename T>
int dev_grow_keep(ktg_ctx *c, T **p, int64_t keep, int64_t count) {
    T *np = nullptr;
    const cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&np), sizeof(T) * std::max<int64_t>(count, 1));
    if (e != cudaSuccess) return ktg::cuda_check(c, e, "cudaMalloc");
    if (*p && keep > 0) {
        const cudaError_t ec = cudaMemcpyAsync(np, *p, sizeof(T) * keep, cudaMemcpyDeviceToDevice,
                                               c->stream);
        if (ec != cudaSuccess) {
            cudaFree(np);
            return ktg::cuda_check(c, ec, "cudaMemcpyAsync");
        }
    }
    if (*p) cudaFree(*p);
    *p = np;
    return KTG_OK;
}

// Room for systems of `rows` rows and `nnz` entries per axis. The arrays
// that hold a system (row pointers, columns, values, diagonal, right-hand
// side) keep their contents when they grow, so an axis installed earlier
// stays valid; the solver scratch is just reallocated.
int reserve_systems(ktg_ctx *c, int64_t rows, int64_t nnz) {
    int rc;
    if (rows > c->sys_cap_n) {
        const int64_t old = c->sys_cap_n;
        for (auto &s : c->sys) {
            if ((rc = dev_grow_keep(c, &s.row_ptr, old > 0 ? old + 1 : 0, rows + 1))) return rc;
            if ((rc = dev_grow_keep(c, &s.diag, old, rows))) return rc;
            if ((rc = dev_grow_keep(c, &s.rhs, old, rows))) return rc;
            if ((rc = dev_alloc(c, &s.r, rows))) return rc;
            if ((rc = dev_alloc(c, &s.z, rows))) return rc;
            if ((rc = dev_alloc(c, &s.p, rows))) return rc;
            if ((rc = dev_alloc(c, &s.ap, rows))) return rc;
            if ((rc = dev_alloc(c, &s.s, rows))) return rc;
            if ((rc = dev_alloc(c, &s.d32, rows))) return rc;
            if ((rc = dev_alloc(c, &s.r32, rows))) return rc;
            if ((rc = dev_alloc(c, &s.z32, rows))) return rc;
            if ((rc = dev_alloc(c, &s.p32, rows))) return rc;
            if ((rc = dev_alloc(c, &s.ap32, rows))) return rc;
            if ((rc = dev_alloc(c, &s.rs32, rows))) return rc;
        }
        if ((rc = dev_alloc(c, &c->x, rows))) return rc;
        if ((rc = dev_alloc(c, &c->y, rows))) return rc;
        if ((rc = dev_alloc(c, &c->ax, rows))) return rc;
        if ((rc = dev_alloc(c, &c->ay, rows))) return rc;
        c->sys_cap_n = rows;
        c->stage_cap = rows;
    }
    if (nnz > c->sys_cap_nnz) {
        const int64_t old = c->sys_cap_nnz;
        for (auto &s : c->sys) {
            if ((rc = dev_grow_keep(c, &s.col, old, nnz))) return rc;
            if ((rc = dev_grow_keep(c, &s.val, old, nnz))) return rc;
            if ((rc = dev_alloc(c, &s.val32, nnz))) return rc;
            if ((rc = dev_alloc(c, &s.s32, nnz))) return rc;
        }
        c->val32_valid = false;
        c->precond_ready = false;
        c->agg_ready = false;
        c->coarse_z_ready = false;
        c->sys_cap_nnz = nnz;
    }
    return KTG_OK;
}

int reserve_partials(ktg_ctx *c, int64_t count) {
    if (count > c->partials_cap) {
        int rc = dev_alloc(c, &c->partials, count);
        if (rc) return rc;
        c->partials_cap = count;
    }
    return KTG_OK;
}

}  // namespace

namespace ktg {

int reserve_system_arrays(ktg_ctx *c, int64_t rows, int64_t nnz) {  // contents kept
    int rc = set_device(c);
    if (rc) return rc;
    return reserve_systems(c, rows, nnz);
}

// The system of one axis from device arrays (row pointers with offsets from
// the row's system start, m entries), copied on the context's stream: what
// ktg_upload_system does for host arrays, for callers that already hold the
// system on this device (the batch's whole-GPU path).
int load_system_device(ktg_ctx *c, int axis, int64_t n, int64_t m, const int32_t *rp,
                       const int32_t *col, const double *val, const double *diag,
                       const double *rhs) {
    if (!c || (axis != 0 && axis != 1) || n < 0 || m < 0 || !rp) return KTG_ERR_ARG;
    if (n > 0x3fffffffll || m > 0x7fffffffll)
        return set_error(c, KTG_ERR_RANGE, "system exceeds 32-bit indices");
    int rc = set_device(c);
    if (rc) return rc;
    if ((rc = reserve_systems(c, n, std::max<int64_t>(m, c->sys_cap_nnz)))) return rc;
    AxisSystem &s = c->sys[axis];
    KTG_CUDA(c, cudaMemcpyAsync(s.row_ptr, rp, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToDevice,
                                c->stream));
    if (m) {
        KTG_CUDA(c, cudaMemcpyAsync(s.col, col, sizeof(int32_t) * m, cudaMemcpyDeviceToDevice,
                                    c->stream));
        KTG_CUDA(c, cudaMemcpyAsync(s.val, val, sizeof(double) * m, cudaMemcpyDeviceToDevice,
                                    c->stream));
    }
    if (n) {
        KTG_CUDA(c, cudaMemcpyAsync(s.diag, diag, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                    c->stream));
        KTG_CUDA(c, cudaMemcpyAsync(s.rhs, rhs, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                    c->stream));
    }
    if (n != c->sys_n) c->axis_valid[1 - axis] = false;
    c->axis_valid[axis] = true;
    c->val32_valid = false;
    c->precond_ready = false;
    c->agg_ready = false;
    c->coarse_z_ready = false;
    c->sys_n = n;
    c->have_system = c->axis_valid[0] && c->axis_valid[1];
    return KTG_OK;
}

}  // namespace ktg

extern "C" {

const char *ktg_version(void) { return "ktplace_b200 0.1 (sm_100a)"; }

int ktg_create(int device, ktg_ctx **out) {
    if (out == nullptr) return KTG_ERR_ARG;
    *out = nullptr;
    ktg_ctx *c = new (std::nothrow) ktg_ctx();
    if (c == nullptr) return KTG_ERR_NOMEM;
    c->device = device;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || device < 0 || device >= count) {
        delete c;
        return KTG_ERR_CUDA;
    }
    int rc = KTG_OK;
    auto fail = [&](int code) {
        ktg_destroy(c);
        return code;
    };
    if ((rc = set_device(c))) return fail(rc);
    if (cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return fail(KTG_ERR_CUDA);
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    if (!coop) return fail(KTG_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(KTG_ERR_CUDA);
    c->stream = c->own_stream;
    if ((rc = dev_alloc(c, &c->counters, 8))) return fail(rc);
    if ((rc = dev_alloc(c, &c->status, 1))) return fail(rc);
    if ((rc = dev_alloc(c, &c->scalars, 8))) return fail(rc);
    if ((rc = dev_alloc(c, &c->info_dev, 1))) return fail(rc);
    if ((rc = dev_alloc(c, &c->minfo_dev, 1))) return fail(rc);
    if (cudaMallocHost(&c->h_minfo, sizeof(ktg_mixed_info)) != cudaSuccess) return fail(KTG_ERR_NOMEM);
    if ((rc = dev_alloc(c, &c->nnz_dev, 2))) return fail(rc);
    if ((rc = reserve_partials(c, 16384))) return fail(rc);
    // stream-ordered (and finished before the handle is returned): the
    // context's stream is non-blocking, so it would not wait for a plain memset
    if (cudaMemsetAsync(c->counters, 0, 8 * sizeof(unsigned), c->stream) != cudaSuccess ||
        cudaMemsetAsync(c->status, 0, sizeof(int), c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
        return fail(KTG_ERR_CUDA);
    if (cudaMallocHost(&c->h_scalars, 8 * sizeof(double)) != cudaSuccess) return fail(KTG_ERR_NOMEM);
    if (cudaMallocHost(&c->h_info, sizeof(ktg_solve_info)) != cudaSuccess) return fail(KTG_ERR_NOMEM);
    if (cudaMallocHost(&c->h_nnz, 2 * sizeof(int64_t)) != cudaSuccess) return fail(KTG_ERR_NOMEM);
    if (cudaMallocHost(&c->h_status, sizeof(int)) != cudaSuccess) return fail(KTG_ERR_NOMEM);
    *out = c;
    return KTG_OK;
}

void ktg_destroy(ktg_ctx *c) {
    if (c == nullptr) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_netlist(c);
    free_systems(c);
    ktg::free_agg(c);
    ktg::free_lal(c);
    dev_free(c->coarse_head_w);
    dev_free(c->coarse_logd);
    dev_free(c->coarse_emb);
    dev_free(c->mixed_trace);
    dev_free(c->hpwl_terms);
    dev_free(c->exact_prod);
    dev_free(c->exact_cpart);
    dev_free(c->partials);
    dev_free(c->counters);
    dev_free(c->status);
    dev_free(c->scalars);
    dev_free(c->info_dev);
    dev_free(c->minfo_dev);
    if (c->h_minfo) cudaFreeHost(c->h_minfo);
    dev_free(c->hist_dev);
    dev_free(c->nnz_dev);
    dev_free(c->avail);
    dev_free(c->occ_fx);
    dev_free(c->occ);
    if (c->h_scalars) cudaFreeHost(c->h_scalars);
    if (c->h_info) cudaFreeHost(c->h_info);
    if (c->h_nnz) cudaFreeHost(c->h_nnz);
    if (c->h_status) cudaFreeHost(c->h_status);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

const char *ktg_last_error(const ktg_ctx *c) { return c ? c->err.c_str() : "null context"; }

int ktg_set_stream(ktg_ctx *c, void *stream) {
    if (!c) return KTG_ERR_ARG;
    c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
    return KTG_OK;
}

int ktg_set_pointer_mode(ktg_ctx *c, int mode) {
    if (!c || (mode != KTG_PTR_HOST && mode != KTG_PTR_DEVICE)) return KTG_ERR_ARG;
    c->ptr_mode = mode;
    return KTG_OK;
}

int64_t ktg_launch_count(const ktg_ctx *c) { return c ? c->launches : 0; }

int ktg_set_option(ktg_ctx *c, const char *key, int64_t value) {
    if (!c || !key) return KTG_ERR_ARG;
    const std::string k(key);
    if (k == "pcg_lanes") {
        if (value != 0 && value != 1 && value != 4 && value != 32)
            return set_error(c, KTG_ERR_ARG, "pcg_lanes must be 0, 1, 4 or 32");
        c->pcg_lanes = static_cast<int>(value);
        return KTG_OK;
    }
    if (k == "mixed_form") {
        if (value != 0 && value != 1) return set_error(c, KTG_ERR_ARG, "mixed_form must be 0 or 1");
        c->mixed_form = static_cast<int>(value);
        return KTG_OK;
    }
    if (k == "precond") {
        if (value != 0 && value != 1 && value != 2)
            return set_error(c, KTG_ERR_ARG, "precond must be 0, 1 or 2");
        c->precond = static_cast<int>(value);
        return KTG_OK;
    }
    if (k == "coarse") {
        if (value < 0 || value > 3) return set_error(c, KTG_ERR_ARG, "coarse must be 0, 1, 2 or 3");
        c->coarse = static_cast<int>(value);
        return KTG_OK;
    }
    if (k == "agg_reuse") {
        if (value < 0 || value > 1000000) return set_error(c, KTG_ERR_ARG, "agg_reuse range");
        c->agg_reuse = static_cast<int>(value);
        return KTG_OK;
    }
    if (k == "hpwl_order") {
        if (value != 0 && value != 2) return set_error(c, KTG_ERR_ARG, "hpwl_order must be 0 or 2");
        c->hpwl_order = static_cast<int>(value);
        return KTG_OK;
    }
    if (k == "mixed_trace") {  // capacity of the mixed solve's phase stamps (0: off)
        if (value < 0 || value > (1 << 20)) return set_error(c, KTG_ERR_ARG, "mixed_trace range");
        dev_free(c->mixed_trace);
        c->mixed_trace_cap = 0;
        if (value > 0) {
            int rc = dev_alloc(c, &c->mixed_trace, value);
            if (rc) return rc;
            KTG_CUDA(c, cudaMemsetAsync(c->mixed_trace, 0, sizeof(unsigned long long) * value,
                                        c->stream));
            c->mixed_trace_cap = static_cast<int32_t>(value);
        }
        return KTG_OK;
    }
    if (k == "pcg_form") {
        if (value < -1 || value > 3)
            return set_error(c, KTG_ERR_ARG, "pcg_form must be -1, 0, 1, 2 or 3");
        c->pcg_form = static_cast<int>(value);
        return KTG_OK;
    }
    if (k == "lal_subtree_cells") {
        if (value < 0 || value > 2048)
            return set_error(c, KTG_ERR_ARG, "lal_subtree_cells must be in [0, 2048]");
        c->lal_subtree_cells = static_cast<int>(value);
        return KTG_OK;
    }
    if (k == "lal_exact_sums") {
        if (value != 0 && value != 1) return set_error(c, KTG_ERR_ARG, "lal_exact_sums must be 0 or 1");
        c->lal_exact_sums = static_cast<int>(value);
        return KTG_OK;
    }
    return set_error(c, KTG_ERR_ARG, "unknown option " + k);
}

int ktg_upload_netlist(ktg_ctx *c, const ktg_netlist_view *nl) {
    if (!c || !nl) return KTG_ERR_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    const int64_t V = nl->num_vertices, n = nl->num_movable, N = nl->num_nets;
    if (V < 0 || n < 0 || N < 0 || n > V) return set_error(c, KTG_ERR_ARG, "negative sizes");
    if ((V > 0 && (!nl->var_of_vertex || !nl->fixed_x || !nl->fixed_y)) ||
        (n > 0 && (!nl->mov_vertex || !nl->pin_start || !nl->width || !nl->height)) ||
        !nl->net_start || (N > 0 && !nl->net_weight))
        return set_error(c, KTG_ERR_ARG, "missing netlist array");
    const int64_t P = nl->net_start[N];
    const int64_t Pm = n > 0 ? nl->pin_start[n] : 0;
    if (P < 0 || Pm < 0 || Pm > P) return set_error(c, KTG_ERR_ARG, "bad pin counts");
    if (P > 0 && (!nl->pin_cell || !nl->off_x || !nl->off_y))
        return set_error(c, KTG_ERR_ARG, "missing pin arrays");
    if (Pm > 0 && (!nl->pin_net || !nl->pin_q)) return set_error(c, KTG_ERR_ARG, "missing pin refs");
    const int64_t lim = 0x7fffffffll;
    if (V > lim || P > lim || N > lim || 2 * n > lim)
        return set_error(c, KTG_ERR_RANGE, "netlist exceeds 32-bit indices");

    // Validate indices on the host once, so no kernel can read out of bounds.
    for (int64_t k = 0; k < N; ++k)
        if (nl->net_start[k + 1] < nl->net_start[k])
            return set_error(c, KTG_ERR_ARG, "net_start not monotone");
    for (int64_t i = 0; i < n; ++i) {
        if (nl->pin_start[i + 1] < nl->pin_start[i])
            return set_error(c, KTG_ERR_ARG, "pin_start not monotone");
        const int32_t v = nl->mov_vertex[i];
        if (v < 0 || v >= V || nl->var_of_vertex[v] != i)
            return set_error(c, KTG_ERR_ARG, "mov_vertex / var_of_vertex disagree");
    }
    std::vector<int32_t> pin_var(P), net_mov(N, 0);
    std::vector<int32_t> net_start32(N + 1), pin_start32(n + 1);
    std::vector<double> net_base(N);
    std::vector<int2> pin_ref(Pm);
    for (int64_t p = 0; p < P; ++p) {
        const int32_t cell = nl->pin_cell[p];
        if (cell < 0 || cell >= V) return set_error(c, KTG_ERR_ARG, "pin_cell out of range");
        const int32_t var = nl->var_of_vertex[cell];
        if (var >= n) return set_error(c, KTG_ERR_ARG, "var_of_vertex out of range");
        pin_var[p] = var < 0 ? -1 : var;
    }
    int64_t cap = 0;
    for (int64_t k = 0; k < N; ++k) {
        net_start32[k] = static_cast<int32_t>(nl->net_start[k]);
        const int64_t deg = nl->net_start[k + 1] - nl->net_start[k];
        // simpl_lss.cc:68: base = weight / (cells.size() - 1), per net
        net_base[k] = nl->net_weight[k] / static_cast<double>(static_cast<uint64_t>(deg - 1));
        int32_t m = 0;
        for (int64_t p = nl->net_start[k]; p < nl->net_start[k + 1]; ++p) m += pin_var[p] >= 0;
        net_mov[k] = m;
        // Bound rows (2) get m-1 movable ends, the others at most 2 each.
        if (m > 0) cap += 4 * static_cast<int64_t>(m);
    }
    net_start32[N] = static_cast<int32_t>(P);
    for (int64_t i = 0; i <= n; ++i) pin_start32[i] = static_cast<int32_t>(nl->pin_start[i]);
    for (int64_t e = 0; e < Pm; ++e) {
        const int32_t k = nl->pin_net[e], q = nl->pin_q[e];
        if (k < 0 || k >= N || q < 0 || q >= nl->net_start[k + 1] - nl->net_start[k])
            return set_error(c, KTG_ERR_ARG, "pin_ref out of range");
        pin_ref[e] = make_int2(k, q);
    }
    for (int64_t i = 0; i < n; ++i)
        for (int64_t e = nl->pin_start[i]; e < nl->pin_start[i + 1]; ++e) {
            const int64_t p = nl->net_start[nl->pin_net[e]] + nl->pin_q[e];
            if (pin_var[p] != i) return set_error(c, KTG_ERR_ARG, "pin_ref does not point to its cell");
        }
    if (cap > lim) return set_error(c, KTG_ERR_RANGE, "B2B systems exceed 32-bit indices");
    std::vector<double> area(n);
    double total_area = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        area[i] = nl->width[i] * nl->height[i];
        total_area += std::fabs(area[i]);
    }
    // Fixed-point shift for the density map: total area * 2^s < 2^61.
    int s = 60;
    if (total_area > 0.0) s = std::min(60, 61 - static_cast<int>(std::ceil(std::log2(total_area + 1.0))));
    s = std::max(s, 0);
    c->fx_scale = std::ldexp(1.0, s);
    // Exact-sum shift of the legalizer: the least q with every area * 2^q an
    // integer and the total * 2^q below 2^52, so that every partial sum of
    // areas, in any order, is exact in double (-1: no such q).
    {
        int q = 0;  // the lowest set bit of every area's significand sets q
        bool ok = true;
        for (int64_t i = 0; ok && i < n; ++i) {
            const double a = area[i];
            if (!(a >= 0.0) || !std::isfinite(a)) ok = false;
            if (!ok || a == 0.0) continue;
            int e;
            const double f = std::frexp(a, &e);  // a = f * 2^e, f in [0.5, 1)
            const auto m = static_cast<uint64_t>(std::ldexp(f, 53));
            const int low_bit = e - 53 + __builtin_ctzll(m);
            q = std::max(q, -low_bit);
        }
        c->area_shift = ok && q <= 60 && std::ldexp(total_area, q) < 4503599627370496.0 ? q : -1;
    }

    KTG_CUDA(c, cudaStreamSynchronize(c->stream));
    free_netlist(c);
    free_systems(c);
    c->V = V;
    c->n = n;
    c->N = N;
    c->P = P;
    c->Pm = Pm;
    c->cap_nnz = std::max<int64_t>(cap, 1);
    if ((rc = dev_alloc(c, &c->var_of_vertex, V))) return rc;
    if ((rc = dev_alloc(c, &c->fixed_x, V))) return rc;
    if ((rc = dev_alloc(c, &c->fixed_y, V))) return rc;
    if ((rc = dev_alloc(c, &c->net_start, N + 1))) return rc;
    if ((rc = dev_alloc(c, &c->pin_cell, P))) return rc;
    if ((rc = dev_alloc(c, &c->pin_var, P))) return rc;
    if ((rc = dev_alloc(c, &c->off_x, P))) return rc;
    if ((rc = dev_alloc(c, &c->off_y, P))) return rc;
    if ((rc = dev_alloc(c, &c->net_base, N))) return rc;
    if ((rc = dev_alloc(c, &c->net_weight, N))) return rc;
    if ((rc = dev_alloc(c, &c->net_mov, N))) return rc;
    if ((rc = dev_alloc(c, &c->pin_start, n + 1))) return rc;
    if ((rc = dev_alloc(c, &c->pin_ref, Pm))) return rc;
    if ((rc = dev_alloc(c, &c->width, n))) return rc;
    if ((rc = dev_alloc(c, &c->height, n))) return rc;
    if ((rc = dev_alloc(c, &c->area, n))) return rc;
    const int64_t bpa = (n + 255) / 256;
    if ((rc = dev_alloc(c, &c->row_cnt, 2 * n))) return rc;
    if ((rc = dev_alloc(c, &c->heavy_rows, 1 + 2 * n))) return rc;
    if ((rc = dev_alloc(c, &c->block_sum, 2 * bpa))) return rc;
    if ((rc = reserve_systems(c, n, c->cap_nnz))) return rc;
    for (auto &s2 : c->sys) {
        if ((rc = dev_alloc(c, &s2.lo, N))) return rc;
        if ((rc = dev_alloc(c, &s2.hi, N))) return rc;
    }
    if ((rc = reserve_partials(c, (N + 255) / 256 + 64))) return rc;
    if ((rc = upload(c, c->var_of_vertex, nl->var_of_vertex, V))) return rc;
    if ((rc = upload(c, c->fixed_x, nl->fixed_x, V))) return rc;
    if ((rc = upload(c, c->fixed_y, nl->fixed_y, V))) return rc;
    if ((rc = upload(c, c->net_start, net_start32.data(), N + 1))) return rc;
    if ((rc = upload(c, c->pin_cell, nl->pin_cell, P))) return rc;
    if ((rc = upload(c, c->pin_var, pin_var.data(), P))) return rc;
    if ((rc = upload(c, c->off_x, nl->off_x, P))) return rc;
    if ((rc = upload(c, c->off_y, nl->off_y, P))) return rc;
    if ((rc = upload(c, c->net_base, net_base.data(), N))) return rc;
    if ((rc = upload(c, c->net_weight, nl->net_weight, N))) return rc;
    if ((rc = upload(c, c->net_mov, net_mov.data(), N))) return rc;
    if ((rc = upload(c, c->pin_start, pin_start32.data(), n + 1))) return rc;
    if ((rc = upload(c, c->pin_ref, pin_ref.data(), Pm))) return rc;
    if ((rc = upload(c, c->width, nl->width, n))) return rc;
    if ((rc = upload(c, c->height, nl->height, n))) return rc;
    if ((rc = upload(c, c->area, area.data(), n))) return rc;
    if ((rc = sync(c))) return rc;
    c->have_netlist = true;
    ++c->netlist_gen;
    c->have_system = false;
    c->sys_n = n;
    return KTG_OK;
}

int ktg_build_b2b(ktg_ctx *c, const double *x, const double *y, double alpha, const double *ax,
                  const double *ay, double floor_x, double floor_y) {
    if (!c) return KTG_ERR_ARG;
    if (!c->have_netlist) return set_error(c, KTG_ERR_STATE, "no netlist uploaded");
    if (c->n > 0 && (!x || !y)) return set_error(c, KTG_ERR_ARG, "null positions");
    if (alpha > 0.0 && c->n > 0 && (!ax || !ay)) return set_error(c, KTG_ERR_ARG, "null anchors");
    int rc = set_device(c);
    if (rc) return rc;
    if ((rc = reserve_systems(c, c->n, c->cap_nnz))) return rc;
    const double *dx = x, *dy = y, *dax = ax, *day = ay;
    if (c->ptr_mode == KTG_PTR_HOST) {
        if ((rc = upload(c, c->x, x, c->n))) return rc;
        if ((rc = upload(c, c->y, y, c->n))) return rc;
        dx = c->x;
        dy = c->y;
        if (alpha > 0.0) {
            if ((rc = upload(c, c->ax, ax, c->n))) return rc;
            if ((rc = upload(c, c->ay, ay, c->n))) return rc;
            dax = c->ax;
            day = c->ay;
        }
    }
    if ((rc = ktg::launch_build_b2b(c, dx, dy, alpha, dax, day, floor_x, floor_y))) return rc;
    c->sys_n = c->n;
    c->have_system = true;
    c->axis_valid[0] = c->axis_valid[1] = true;
    c->val32_valid = false;
    c->precond_ready = false;
    c->agg_ready = false;
    c->coarse_z_ready = false;
    if (c->ptr_mode == KTG_PTR_HOST) {
        const int st = device_status(c);
        if (st < 0) return st;
        if (st != 0) return set_error(c, st, "B2B system exceeds its capacity");
    }
    return KTG_OK;
}

int ktg_build_b2b_kraftwerk2(ktg_ctx *c, const double *x, const double *y, int with_rhs,
                             double floor_x, double floor_y) {
    if (!c) return KTG_ERR_ARG;
    if (!c->have_netlist) return set_error(c, KTG_ERR_STATE, "no netlist uploaded");
    if (c->n > 0 && (!x || !y)) return set_error(c, KTG_ERR_ARG, "null positions");
    int rc = set_device(c);
    if (rc) return rc;
    if ((rc = reserve_systems(c, c->n, c->cap_nnz))) return rc;
    const double *dx = x, *dy = y;
    if (c->ptr_mode == KTG_PTR_HOST) {
        if ((rc = upload(c, c->x, x, c->n))) return rc;
        if ((rc = upload(c, c->y, y, c->n))) return rc;
        dx = c->x;
        dy = c->y;
    }
    if ((rc = ktg::launch_build_kraftwerk2(c, dx, dy, with_rhs != 0, floor_x, floor_y))) return rc;
    c->sys_n = c->n;
    c->have_system = true;
    c->axis_valid[0] = c->axis_valid[1] = true;
    c->val32_valid = false;
    c->precond_ready = false;
    c->agg_ready = false;
    c->coarse_z_ready = false;
    if (c->ptr_mode == KTG_PTR_HOST) {
        const int st = device_status(c);
        if (st < 0) return st;
        if (st != 0) return set_error(c, st, "Kraftwerk2 system exceeds its capacity");
    }
    return KTG_OK;
}

int ktg_kraftwerk2_adjust(ktg_ctx *c, const double *move_weight, const double *toward_x,
                          const double *toward_y, double diag_floor) {
    if (!c) return KTG_ERR_ARG;
    if (!c->have_system) return set_error(c, KTG_ERR_STATE, "no system to adjust");
    if (move_weight && (!toward_x || !toward_y))
        return set_error(c, KTG_ERR_ARG, "move_weight needs toward_x and toward_y");
    int rc = set_device(c);
    if (rc) return rc;
    const int64_t n = c->sys_n;
    const double *mw = move_weight, *tx = toward_x, *ty = toward_y;
    if (move_weight && c->ptr_mode == KTG_PTR_HOST) {
        // staging: ax / ay hold the two toward vectors, x holds the weights
        if ((rc = upload(c, c->ax, toward_x, n))) return rc;
        if ((rc = upload(c, c->ay, toward_y, n))) return rc;
        if ((rc = upload(c, c->x, move_weight, n))) return rc;
        mw = c->x;
        tx = c->ax;
        ty = c->ay;
    }
    if ((rc = ktg::launch_kraftwerk2_adjust(c, mw, tx, ty, diag_floor))) return rc;
    c->val32_valid = false;
    c->precond_ready = false;
    c->agg_ready = false;
    c->coarse_z_ready = false;
    if (c->ptr_mode == KTG_PTR_HOST) return sync(c);
    return KTG_OK;
}

int ktg_build_star(ktg_ctx *c, int64_t *size) {
    if (!c || !size) return KTG_ERR_ARG;
    if (!c->have_netlist) return set_error(c, KTG_ERR_STATE, "no netlist uploaded");
    int rc = set_device(c);
    if (rc) return rc;
    int64_t rows = 0;
    if ((rc = ktg::build_star(c, &rows, reserve_systems))) return rc;
    c->sys_n = rows;
    c->have_system = true;
    c->axis_valid[0] = c->axis_valid[1] = true;
    c->val32_valid = false;
    c->precond_ready = false;
    c->agg_ready = false;
    c->coarse_z_ready = false;
    *size = rows;
    return KTG_OK;
}

int ktg_build_hpwl(ktg_ctx *c, double *out) {
    if (!c || !out) return KTG_ERR_ARG;
    if (!c->have_system) return set_error(c, KTG_ERR_STATE, "no B2B build yet");
    int rc = set_device(c);
    if (rc) return rc;
    if (c->ptr_mode == KTG_PTR_DEVICE) {
        KTG_CUDA(c, cudaMemcpyAsync(out, c->scalars + 0, sizeof(double), cudaMemcpyDeviceToDevice,
                                    c->stream));
        return KTG_OK;
    }
    KTG_CUDA(c, cudaMemcpyAsync(c->h_scalars, c->scalars, sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
    if ((rc = sync(c))) return rc;
    *out = c->h_scalars[0];
    return KTG_OK;
}

int ktg_system_info(ktg_ctx *c, int axis, int64_t *n, int64_t *nnz) {
    if (!c || (axis != 0 && axis != 1)) return KTG_ERR_ARG;
    if (!c->axis_valid[axis]) return set_error(c, KTG_ERR_STATE, "no system for this axis");
    int rc = set_device(c);
    if (rc) return rc;
    int32_t m = 0;
    KTG_CUDA(c, cudaMemcpyAsync(&m, c->sys[axis].row_ptr + c->sys_n, sizeof(int32_t),
                                cudaMemcpyDeviceToHost, c->stream));
    if ((rc = sync(c))) return rc;
    if (n) *n = c->sys_n;
    if (nnz) *nnz = m;
    return KTG_OK;
}

int ktg_download_system(ktg_ctx *c, int axis, int64_t *row_ptr, int32_t *col, double *val,
                        double *diag, double *rhs) {
    int64_t n = 0, m = 0;
    int rc = ktg_system_info(c, axis, &n, &m);
    if (rc) return rc;
    const ktg::AxisSystem &s = c->sys[axis];
    std::vector<int32_t> rp(n + 1);
    KTG_CUDA(c, cudaMemcpy(rp.data(), s.row_ptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost));
    if (row_ptr)
        for (int64_t i = 0; i <= n; ++i) row_ptr[i] = rp[i];
    if (col && m) KTG_CUDA(c, cudaMemcpy(col, s.col, sizeof(int32_t) * m, cudaMemcpyDeviceToHost));
    if (val && m) KTG_CUDA(c, cudaMemcpy(val, s.val, sizeof(double) * m, cudaMemcpyDeviceToHost));
    if (diag && n) KTG_CUDA(c, cudaMemcpy(diag, s.diag, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (rhs && n) KTG_CUDA(c, cudaMemcpy(rhs, s.rhs, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return KTG_OK;
}

int ktg_download_bound_pins(ktg_ctx *c, int axis, uint32_t *lo, uint32_t *hi) {
    if (!c || (axis != 0 && axis != 1)) return KTG_ERR_ARG;
    if (!c->have_netlist) return set_error(c, KTG_ERR_STATE, "no netlist uploaded");
    int rc = set_device(c);
    if (rc) return rc;
    if ((rc = sync(c))) return rc;
    if (lo && c->N)
        KTG_CUDA(c, cudaMemcpy(lo, c->sys[axis].lo, sizeof(uint32_t) * c->N, cudaMemcpyDeviceToHost));
    if (hi && c->N)
        KTG_CUDA(c, cudaMemcpy(hi, c->sys[axis].hi, sizeof(uint32_t) * c->N, cudaMemcpyDeviceToHost));
    return KTG_OK;
}

int ktg_upload_system(ktg_ctx *c, int axis, int64_t n, const int64_t *row_ptr, const int32_t *col,
                      const double *val, const double *diag, const double *rhs) {
    if (!c || (axis != 0 && axis != 1) || n < 0 || !row_ptr) return KTG_ERR_ARG;
    if (n > 0 && (!diag || !rhs)) return KTG_ERR_ARG;
    const int64_t m = row_ptr[n];
    if (m < 0 || m > 0x7fffffffll || n > 0x3fffffffll)
        return set_error(c, KTG_ERR_RANGE, "system exceeds 32-bit indices");
    if (m > 0 && (!col || !val)) return KTG_ERR_ARG;
    std::vector<int32_t> rp(n + 1);
    for (int64_t i = 0; i <= n; ++i) {
        if (row_ptr[i] < 0 || (i > 0 && row_ptr[i] < row_ptr[i - 1]))
            return set_error(c, KTG_ERR_ARG, "row_ptr not monotone");
        rp[i] = static_cast<int32_t>(row_ptr[i]);
    }
    for (int64_t e = 0; e < m; ++e)
        if (col[e] < 0 || col[e] >= n) return set_error(c, KTG_ERR_ARG, "col out of range");
    int rc = set_device(c);
    if (rc) return rc;
    if ((rc = sync(c))) return rc;
    if ((rc = reserve_systems(c, n, std::max<int64_t>(m, c->sys_cap_nnz)))) return rc;
    ktg::AxisSystem &s = c->sys[axis];
    if ((rc = upload(c, s.row_ptr, rp.data(), n + 1))) return rc;
    if ((rc = upload(c, s.col, col, m))) return rc;
    if ((rc = upload(c, s.val, val, m))) return rc;
    if ((rc = upload(c, s.diag, diag, n))) return rc;
    if ((rc = upload(c, s.rhs, rhs, n))) return rc;
    if ((rc = sync(c))) return rc;
    if (n != c->sys_n) c->axis_valid[1 - axis] = false;
    c->axis_valid[axis] = true;
    c->val32_valid = false;
    c->precond_ready = false;
    c->agg_ready = false;
    c->coarse_z_ready = false;
    c->sys_n = n;
    c->have_system = c->axis_valid[0] && c->axis_valid[1];
    return KTG_OK;
}

int ktg_solve(ktg_ctx *c, double *x, double *y, double tol, int64_t max_iter, ktg_solve_info *info,
              double *hist_x, double *hist_y, int64_t hist_cap) {
    if (!c) return KTG_ERR_ARG;
    if (!c->have_system) return set_error(c, KTG_ERR_STATE, "no system to solve");
    if (c->sys_n > 0 && (!x || !y)) return set_error(c, KTG_ERR_ARG, "null positions");
    if (max_iter < 0 || hist_cap < 0) return set_error(c, KTG_ERR_ARG, "negative count");
    if (hist_cap > 0 && !hist_x && !hist_y) hist_cap = 0;
    int rc = set_device(c);
    if (rc) return rc;
    const int64_t n = c->sys_n;
    if (c->ptr_mode == KTG_PTR_DEVICE) {
        if ((rc = ktg::launch_solve(c, x, y, tol, max_iter, info ? info : c->info_dev, hist_x,
                                    hist_y, hist_cap)))
            return rc;
        return KTG_OK;
    }
    if (hist_cap > c->hist_cap_dev) {
        if ((rc = dev_alloc(c, &c->hist_dev, 2 * hist_cap))) return rc;
        c->hist_cap_dev = hist_cap;
    }
    if ((rc = upload(c, c->x, x, n))) return rc;
    if ((rc = upload(c, c->y, y, n))) return rc;
    if ((rc = ktg::launch_solve(c, c->x, c->y, tol, max_iter, c->info_dev,
                                hist_x ? c->hist_dev : nullptr,
                                hist_y ? c->hist_dev + hist_cap : nullptr, hist_cap)))
        return rc;
    KTG_CUDA(c, cudaMemcpyAsync(x, c->x, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    KTG_CUDA(c, cudaMemcpyAsync(y, c->y, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    KTG_CUDA(c, cudaMemcpyAsync(c->h_info, c->info_dev, sizeof(ktg_solve_info),
                                cudaMemcpyDeviceToHost, c->stream));
    if ((rc = sync(c))) return rc;
    const ktg_solve_info inf = *c->h_info;
    if (info) *info = inf;
    if (inf.status != KTG_OK) return set_error(c, inf.status, "PCG barrier wait timed out");
    if (hist_cap > 0) {
        const int64_t k = std::min<int64_t>(inf.iters, hist_cap);
        if (hist_x && k)
            KTG_CUDA(c, cudaMemcpy(hist_x, c->hist_dev, sizeof(double) * k, cudaMemcpyDeviceToHost));
        if (hist_y && k)
            KTG_CUDA(c, cudaMemcpy(hist_y, c->hist_dev + hist_cap, sizeof(double) * k,
                                   cudaMemcpyDeviceToHost));
    }
    return KTG_OK;
}

namespace {
__global__ void k_copy_fp64_iters(const ktg_solve_info *s, ktg_mixed_info *m) {
    m->fp64_iters_x = s->iters_x;
    m->fp64_iters_y = s->iters_y;
    if (s->status != KTG_OK) m->status = s->status;
    m->resid_x = s->iters_x > 0 ? s->resid_x : m->resid_x;
    m->resid_y = s->iters_y > 0 ? s->resid_y : m->resid_y;
}
}  // namespace

int ktg_solve_mixed(ktg_ctx *c, double *x, double *y, double tol, double inner_tol,
                    int64_t max_inner, int32_t max_outer, ktg_mixed_info *info, double *hist_x,
                    double *hist_y, int64_t hist_cap) {
    if (!c) return KTG_ERR_ARG;
    if (!c->have_system) return set_error(c, KTG_ERR_STATE, "no system to solve");
    if (c->sys_n > 0 && (!x || !y)) return set_error(c, KTG_ERR_ARG, "null positions");
    if (!(inner_tol > 0.0 && inner_tol < 1.0) || max_inner < 0 || max_outer < 0 || hist_cap < 0)
        return set_error(c, KTG_ERR_ARG, "bad mixed-precision parameters");
    if (hist_cap > 0 && !hist_x && !hist_y) hist_cap = 0;
    int rc = set_device(c);
    if (rc) return rc;
    const int64_t n = c->sys_n;
    if (c->ptr_mode == KTG_PTR_DEVICE) {
        ktg_mixed_info *mi = info ? info : c->minfo_dev;
        if ((rc = ktg::launch_solve_mixed(c, x, y, tol, inner_tol, max_inner, max_outer, mi,
                                          hist_x, hist_y, hist_cap)))
            return rc;
        // FP64 pass: finishes a stalled or unfinished axis; every block returns
        // at once (before any work) when the mixed result says both converged.
        c->pcg_gate = mi;
        rc = ktg::launch_solve(c, x, y, tol, max_inner, c->info_dev, nullptr, nullptr, 0);
        c->pcg_gate = nullptr;
        if (rc) return rc;
        k_copy_fp64_iters<<<1, 1, 0, c->stream>>>(c->info_dev, mi);
        ++c->launches;
        KTG_CUDA(c, cudaGetLastError());
        return KTG_OK;
    }
    if (hist_cap > c->hist_cap_dev) {
        if ((rc = dev_alloc(c, &c->hist_dev, 2 * hist_cap))) return rc;
        c->hist_cap_dev = hist_cap;
    }
    if ((rc = upload(c, c->x, x, n))) return rc;
    if ((rc = upload(c, c->y, y, n))) return rc;
    if ((rc = ktg::launch_solve_mixed(c, c->x, c->y, tol, inner_tol, max_inner, max_outer,
                                      c->minfo_dev, hist_x ? c->hist_dev : nullptr,
                                      hist_y ? c->hist_dev + hist_cap : nullptr, hist_cap)))
        return rc;
    KTG_CUDA(c, cudaMemcpyAsync(c->h_minfo, c->minfo_dev, sizeof(ktg_mixed_info),
                                cudaMemcpyDeviceToHost, c->stream));
    if ((rc = sync(c))) return rc;
    ktg_mixed_info inf = *c->h_minfo;
    if (inf.status != KTG_OK) return set_error(c, inf.status, "mixed PCG barrier wait timed out");
    const bool unfinished = (inf.stalled != 0) || inf.resid_x > tol || inf.resid_y > tol;
    if (unfinished) {
        if ((rc = ktg::launch_solve(c, c->x, c->y, tol, max_inner, c->info_dev, nullptr, nullptr, 0)))
            return rc;
        KTG_CUDA(c, cudaMemcpyAsync(c->h_info, c->info_dev, sizeof(ktg_solve_info),
                                    cudaMemcpyDeviceToHost, c->stream));
        if ((rc = sync(c))) return rc;
        const ktg_solve_info s = *c->h_info;
        if (s.status != KTG_OK) return set_error(c, s.status, "PCG barrier wait timed out");
        inf.fp64_iters_x = s.iters_x;
        inf.fp64_iters_y = s.iters_y;
        if (s.iters_x > 0) inf.resid_x = s.resid_x;
        if (s.iters_y > 0) inf.resid_y = s.resid_y;
    }
    KTG_CUDA(c, cudaMemcpyAsync(x, c->x, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    KTG_CUDA(c, cudaMemcpyAsync(y, c->y, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    if ((rc = sync(c))) return rc;
    if (info) *info = inf;
    if (hist_cap > 0) {
        const int64_t k = std::min<int64_t>(std::max(inf.outer_x, inf.outer_y), hist_cap);
        if (hist_x && k)
            KTG_CUDA(c, cudaMemcpy(hist_x, c->hist_dev, sizeof(double) * k, cudaMemcpyDeviceToHost));
        if (hist_y && k)
            KTG_CUDA(c, cudaMemcpy(hist_y, c->hist_dev + hist_cap, sizeof(double) * k,
                                   cudaMemcpyDeviceToHost));
    }
    return KTG_OK;
}

int ktg_download_aggregates(ktg_ctx *c, int32_t *order, int32_t *meta, float *minv) {
    if (!c) return KTG_ERR_ARG;
    if (!c->have_system) return set_error(c, KTG_ERR_STATE, "no system to aggregate");
    int rc = set_device(c);
    if (rc) return rc;
    if (!c->agg_ready && (rc = ktg::build_agg(c))) return rc;
    const int64_t rows = 2 * c->sys_n;
    const ktg::AggState *g = c->agg;
    if (rows > 0) {
        if (order)
            KTG_CUDA(c, cudaMemcpyAsync(order, g->order, sizeof(int32_t) * rows,
                                        cudaMemcpyDeviceToHost, c->stream));
        if (meta)
            KTG_CUDA(c, cudaMemcpyAsync(meta, g->meta, sizeof(int32_t) * rows,
                                        cudaMemcpyDeviceToHost, c->stream));
        if (minv)
            KTG_CUDA(c, cudaMemcpyAsync(minv, g->minv, sizeof(float) * 8 * rows,
                                        cudaMemcpyDeviceToHost, c->stream));
    }
    return sync(c);
}

int ktg_download_mixed_trace(ktg_ctx *c, uint64_t *out, int64_t cap) {
    if (!c || !out || cap < 0) return KTG_ERR_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    const int64_t k = std::min<int64_t>(cap, c->mixed_trace_cap);
    if (k > 0)
        KTG_CUDA(c, cudaMemcpyAsync(out, c->mixed_trace, sizeof(uint64_t) * k,
                                    cudaMemcpyDeviceToHost, c->stream));
    return sync(c);
}

int ktg_download_coarse(ktg_ctx *c, float *z, float *az, double *einv) {
    if (!c) return KTG_ERR_ARG;
    if (!c->have_system) return set_error(c, KTG_ERR_STATE, "no system to aggregate");
    if (c->coarse <= 0) return set_error(c, KTG_ERR_STATE, "coarse option is 0");
    if (c->coarse == 3 && !c->coarse_z_ready)
        return set_error(c, KTG_ERR_STATE, "learned coarse vector not prepared");
    int rc = set_device(c);
    if (rc) return rc;
    if (!c->agg_ready && (rc = ktg::build_agg(c))) return rc;
    if ((rc = ktg::agg_coarse_setup(c, c->coarse))) return rc;
    const int64_t rows = 2 * c->sys_n;
    const ktg::AggState *g = c->agg;
    if (rows > 0 && (z || az)) {
        std::vector<float2> h(rows);
        KTG_CUDA(c, cudaMemcpyAsync(h.data(), g->zaz, sizeof(float2) * rows,
                                    cudaMemcpyDeviceToHost, c->stream));
        if ((rc = sync(c))) return rc;
        for (int64_t k = 0; k < rows; ++k) {
            if (z) z[k] = h[k].x;
            if (az) az[k] = h[k].y;
        }
    }
    if (einv)
        KTG_CUDA(c, cudaMemcpyAsync(einv, g->coarse_einv, 2 * sizeof(double),
                                    cudaMemcpyDeviceToHost, c->stream));
    return sync(c);
}

int ktg_hpwl(ktg_ctx *c, const double *x, const double *y, double *out) {
    if (!c || !out) return KTG_ERR_ARG;
    if (!c->have_netlist) return set_error(c, KTG_ERR_STATE, "no netlist uploaded");
    if (c->n > 0 && (!x || !y)) return set_error(c, KTG_ERR_ARG, "null positions");
    int rc = set_device(c);
    if (rc) return rc;
    if (c->ptr_mode == KTG_PTR_DEVICE) return ktg::launch_hpwl(c, x, y, out);
    if ((rc = reserve_systems(c, c->n, 0))) return rc;
    if ((rc = upload(c, c->x, x, c->n))) return rc;
    if ((rc = upload(c, c->y, y, c->n))) return rc;
    if ((rc = ktg::launch_hpwl(c, c->x, c->y, c->scalars + 1))) return rc;
    KTG_CUDA(c, cudaMemcpyAsync(c->h_scalars + 1, c->scalars + 1, sizeof(double),
                                cudaMemcpyDeviceToHost, c->stream));
    if ((rc = sync(c))) return rc;
    *out = c->h_scalars[1];
    return KTG_OK;
}

int ktg_spmv(ktg_ctx *c, int32_t axis, const double *in, double *out) {
    if (!c) return KTG_ERR_ARG;
    if (!c->have_system) return set_error(c, KTG_ERR_STATE, "no system built");
    if (axis != 0 && axis != 1) return set_error(c, KTG_ERR_ARG, "axis must be 0 or 1");
    if (c->sys_n > 0 && (!in || !out)) return set_error(c, KTG_ERR_ARG, "null vector");
    const int64_t n = c->sys_n;
    // other rows gather `in` while `out` is written: the two may not overlap
    // on the device (host buffers are staged separately, so they may)
    if (c->ptr_mode == KTG_PTR_DEVICE && n > 0 && in < out + n && out < in + n)
        return set_error(c, KTG_ERR_ARG, "ktg_spmv: in and out overlap");
    int rc = set_device(c);
    if (rc) return rc;
    if (c->ptr_mode == KTG_PTR_DEVICE) return ktg::launch_spmv(c, axis, in, out);
    if ((rc = upload(c, c->x, in, n))) return rc;
    if ((rc = ktg::launch_spmv(c, axis, c->x, c->y))) return rc;
    if (n > 0)
        KTG_CUDA(c, cudaMemcpyAsync(out, c->y, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                    c->stream));
    return sync(c);
}

int ktg_set_grid(ktg_ctx *c, const ktg_grid_view *g) {
    if (!c || !g) return KTG_ERR_ARG;
    if (g->nx <= 0 || g->ny <= 0 || !g->avail || !(g->dx > 0.0) || !(g->dy > 0.0))
        return set_error(c, KTG_ERR_ARG, "bad grid");
    if (g->nx * g->ny > 0x7fffffffll || g->nx > 0x7fffffffll || g->ny > 0x7fffffffll)
        return set_error(c, KTG_ERR_RANGE, "grid exceeds 32-bit indices");
    int rc = set_device(c);
    if (rc) return rc;
    const int64_t bins = g->nx * g->ny;
    if ((rc = sync(c))) return rc;
    if (bins > c->bins_cap) {
        if ((rc = dev_alloc(c, &c->avail, bins))) return rc;
        if ((rc = dev_alloc(c, &c->occ_fx, bins))) return rc;
        if ((rc = dev_alloc(c, &c->occ, bins))) return rc;
        c->bins_cap = bins;
    }
    if ((rc = reserve_partials(c, (bins + 255) / 256 + 64))) return rc;
    KTG_CUDA(c, cudaMemsetAsync(c->occ_fx, 0, sizeof(unsigned long long) * bins, c->stream));
    if ((rc = upload(c, c->avail, g->avail, bins))) return rc;
    c->avail_host.resize(static_cast<size_t>(bins));
    KTG_CUDA(c, cudaMemcpyAsync(c->avail_host.data(), c->avail, sizeof(double) * bins,
                                cudaMemcpyDeviceToHost, c->stream));
    if ((rc = sync(c))) return rc;
    c->nx = g->nx;
    c->ny = g->ny;
    c->origin_x = g->origin_x;
    c->origin_y = g->origin_y;
    c->dx = g->dx;
    c->dy = g->dy;
    c->total_avail = g->total_avail;
    c->density_limit = std::clamp(g->density_limit, 0.05, 1.0);
    c->have_grid = true;
    return KTG_OK;
}

int ktg_occupancy(ktg_ctx *c, const double *x, const double *y, double *occ, double *overflow) {
    if (!c || !overflow) return KTG_ERR_ARG;
    if (!c->have_netlist) return set_error(c, KTG_ERR_STATE, "no netlist uploaded");
    if (!c->have_grid) return set_error(c, KTG_ERR_STATE, "no grid installed");
    if (c->n > 0 && (!x || !y)) return set_error(c, KTG_ERR_ARG, "null positions");
    int rc = set_device(c);
    if (rc) return rc;
    if (c->ptr_mode == KTG_PTR_DEVICE) return ktg::launch_occupancy(c, x, y, occ, overflow);
    if ((rc = reserve_systems(c, c->n, 0))) return rc;
    if ((rc = upload(c, c->x, x, c->n))) return rc;
    if ((rc = upload(c, c->y, y, c->n))) return rc;
    if ((rc = ktg::launch_occupancy(c, c->x, c->y, occ ? c->occ : nullptr, c->scalars + 2)))
        return rc;
    const int64_t bins = c->nx * c->ny;
    if (occ)
        KTG_CUDA(c, cudaMemcpyAsync(occ, c->occ, sizeof(double) * bins, cudaMemcpyDeviceToHost,
                                    c->stream));
    KTG_CUDA(c, cudaMemcpyAsync(c->h_scalars + 2, c->scalars + 2, sizeof(double),
                                cudaMemcpyDeviceToHost, c->stream));
    if ((rc = sync(c))) return rc;
    *overflow = c->h_scalars[2];
    return KTG_OK;
}

int ktg_set_free_space(ktg_ctx *c, int64_t num_rows, const double *row_y,
                       const int64_t *row_span, const double *spans, int64_t num_obstacles,
                       const double *obstacles, const double *die) {
    if (!c || !die || num_rows < 0 || num_obstacles < 0) return KTG_ERR_ARG;
    if (num_rows > 0 && (!row_y || !row_span)) return set_error(c, KTG_ERR_ARG, "null rows");
    if (num_obstacles > 0 && !obstacles) return set_error(c, KTG_ERR_ARG, "null obstacles");
    if (num_rows > 0x7fffffffll || num_obstacles > 0x7fffffffll)
        return set_error(c, KTG_ERR_RANGE, "free space exceeds 32-bit indices");
    const int64_t zero = 0;
    const int64_t *rs = num_rows > 0 ? row_span : &zero;
    if (rs[0] != 0) return set_error(c, KTG_ERR_ARG, "row_span[0] must be 0");
    for (int64_t r = 0; r < num_rows; ++r) {
        if (rs[r + 1] < rs[r]) return set_error(c, KTG_ERR_ARG, "row_span not ascending");
        if (r > 0 && row_y[2 * r] < row_y[2 * r - 2])
            return set_error(c, KTG_ERR_ARG, "rows not sorted by their bottom edge");
    }
    if (rs[num_rows] > 0 && !spans) return set_error(c, KTG_ERR_ARG, "null spans");
    int rc = set_device(c);
    if (rc) return rc;
    if ((rc = sync(c))) return rc;
    if ((rc = ktg::set_free_space(c, num_rows, row_y, rs, spans, num_obstacles, obstacles, die)))
        return rc;
    c->have_free_space = true;
    return KTG_OK;
}

int ktg_lal(ktg_ctx *c, double *x, double *y, int32_t max_level, int32_t min_cells_to_split,
            double stripe_area_fraction) {
    if (!c) return KTG_ERR_ARG;
    if (!c->have_netlist) return set_error(c, KTG_ERR_STATE, "no netlist uploaded");
    if (!c->have_grid) return set_error(c, KTG_ERR_STATE, "no grid installed");
    if (!c->have_free_space) return set_error(c, KTG_ERR_STATE, "no free space installed");
    if (c->n > 0 && (!x || !y)) return set_error(c, KTG_ERR_ARG, "null positions");
    if (max_level < 1 || min_cells_to_split < 0 || !(stripe_area_fraction > 0.0))
        return set_error(c, KTG_ERR_ARG, "bad legalization options");
    int rc = set_device(c);
    if (rc) return rc;
    double *dx = x, *dy = y;
    if (c->ptr_mode == KTG_PTR_HOST) {
        if ((rc = reserve_systems(c, c->n, 0))) return rc;
        if ((rc = upload(c, c->x, x, c->n))) return rc;
        if ((rc = upload(c, c->y, y, c->n))) return rc;
        dx = c->x;
        dy = c->y;
    }
    if ((rc = ktg::launch_lal(c, dx, dy, max_level, min_cells_to_split, stripe_area_fraction)))
        return rc;
    if (c->ptr_mode == KTG_PTR_HOST && c->n > 0) {
        KTG_CUDA(c, cudaMemcpyAsync(x, dx, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
        KTG_CUDA(c, cudaMemcpyAsync(y, dy, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
    }
    const int st = device_status(c);
    if (st < 0) return st;
    if (st != 0) return set_error(c, st, "legalization stripes exceed their capacity");
    return KTG_OK;
}

int ktg_lal_stats(ktg_ctx *c, double *out, int32_t count) {
    if (!c || !out || count < 0) return KTG_ERR_ARG;
    return ktg::lal_stats(c, out, count);
}

}  // extern "C"
