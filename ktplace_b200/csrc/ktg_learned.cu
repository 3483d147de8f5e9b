// Learned sparse approximate inverse for the PCG (sm_100a): network
// inference, training (forward + backward + Adam) and preparation of the
// preconditioner values, all in hand-written kernels.
//
// Preconditioner (SPD by construction, on A's own sparsity pattern):
//   M = D^-1/2 (I + S) D^-1/2,  s_e = t_e |a_e| / sqrt(d_i d_j),
//   t_e = clamp(tanh(<p_i, p_j> / 4), -0.999, 0.999)
// |S| <= 0.999 D^-1/2 |A_off| D^-1/2 entrywise, whose spectral radius is at
// most 1 for the diagonally dominant M-matrices B2B builds, so I + S is SPD
// (t = 1 would be the first-order Neumann preconditioner). p (16 per cell)
// comes from a 3-layer message-passing network over the cell-net bipartite
// graph (hidden width 64, mean aggregation, ReLU):
//   h0 = relu(x W_in + b_in),  x = 8 per-cell features of the system
//   per layer: m = mean_cells->net(h), e = relu(m Wa + ba),
//              g = mean_nets->cell(e), h = relu(h Wb + g Wc + bb)
//   p = h P
// Dense layers keep FP32 master weights and use BF16 copies on the tensor
// cores: tcgen05.mma with the FP32 accumulator in tensor memory (default),
// or the older warp-level mma.sync m16n8k16; an FP32 CUDA-core path of the
// same layers exists for gradient checks. Training minimises
//   L = mean over K Rademacher probes v of ||M A v - v||^2 / n
// on systems the GPU SimPL loop produces. Every reduction (weight gradients,
// loss) runs in a fixed order, so training is reproducible run to run.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <new>
#include <string>
#include <vector>

#include "ktg_coarse_head.cuh"
#include "ktg_common.cuh"
#include "ktg_context.h"
#include "ktplace_b200.h"

namespace ktg {
namespace learned {

constexpr int HID = 64;
constexpr int PROJ = 16;
constexpr int NFEAT = 8;
constexpr int LAYERS = 3;
// coarse-vector head: input = p (PROJ), coupling share, log diag
constexpr int HEAD_IN = PROJ + 2;
constexpr int HEAD_H = 16;
static_assert(PROJ == ktg::kCoarseProj && HEAD_IN == ktg::kCoarseIn && HEAD_H == ktg::kCoarseHid,
              "the coarse head's shape is shared with the aggregation build");
constexpr int kMaxVec = 4;  // test vectors per coarse loss
// softplus^-1(1): the head's output bias at initialisation, so that the
// untrained head gives the constant coarse vector
constexpr double kSoftplusInvOne = 0.5413248546129181;

// Parameter layout (FP32 master, same order as oracle/learned_ref.py).
struct Layout {
    int64_t W_in, b_in, Wa[LAYERS], ba[LAYERS], Wb[LAYERS], Wc[LAYERS], bb[LAYERS], P;
    int64_t Wh, bh, wz, bz, total;
};

inline Layout layout() {
    Layout L{};
    int64_t o = 0;
    L.W_in = o; o += NFEAT * HID;
    L.b_in = o; o += HID;
    for (int l = 0; l < LAYERS; ++l) {
        L.Wa[l] = o; o += HID * HID;
        L.ba[l] = o; o += HID;
        L.Wb[l] = o; o += HID * HID;
        L.Wc[l] = o; o += HID * HID;
        L.bb[l] = o; o += HID;
    }
    L.P = o; o += HID * PROJ;
    L.Wh = o; o += HEAD_IN * HEAD_H;
    L.bh = o; o += HEAD_H;
    L.wz = o; o += HEAD_H;
    L.bz = o; o += 1;
    L.total = o;
    return L;
}

// ---------------------------------------------------------------------------
// features
// ---------------------------------------------------------------------------
__global__ void k_logd_sum(const double *diag, int32_t n, double *partials, unsigned *ticket,
                           double *out) {
    __shared__ double scratch[40];
    double v = 0.0;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        v += log(diag[i]);
    const double bs = block_sum(v, scratch);
    if (threadIdx.x == 0) __stcg(partials + blockIdx.x, bs);
    if (last_block_done(ticket)) {
        const double t = sum_partials(partials, gridDim.x, scratch);
        if (threadIdx.x == 0) *out = n > 0 ? t / n : 0.0;
    }
}

__global__ void k_features(const int32_t *rp, const int32_t *col, const double *val,
                           const double *diag, const int32_t *pin_start, int32_t n,
                           const double *logd_mean, float *x) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = diag[i];
    double rowabs = 0.0, rowmax = 0.0;
    for (int32_t e = rp[i]; e < rp[i + 1]; ++e) {
        const double a = fabs(val[e]);
        rowabs += a;
        rowmax = a > rowmax ? a : rowmax;
    }
    const double nnz = static_cast<double>(rp[i + 1] - rp[i]);
    const double npins = static_cast<double>(pin_start[i + 1] - pin_start[i]);
    float *xi = x + static_cast<int64_t>(i) * NFEAT;
    xi[0] = 1.0f;
    xi[1] = static_cast<float>(log(d) - *logd_mean);
    xi[2] = static_cast<float>((d - rowabs) / d);
    xi[3] = static_cast<float>(nnz / 16.0);
    xi[4] = static_cast<float>(npins / 8.0);
    xi[5] = static_cast<float>(rowabs / d);
    xi[6] = static_cast<float>(rowmax / d);
    xi[7] = static_cast<float>(log1p(nnz) / 4.0);
}

// ---------------------------------------------------------------------------
// mean aggregations over the bipartite graph (one warp per output row,
// two channels per lane; sums in pin order: deterministic)
// ---------------------------------------------------------------------------
// m[k] = (1/cnt_k) sum over movable pins of net k of h[cell]
__global__ void k_cells_to_nets(const int32_t *net_start, const int32_t *pin_var,
                                const int32_t *net_mov, int32_t N, const float *h, float *m) {
    const int32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (k >= N) return;
    float a0 = 0.f, a1 = 0.f;
    for (int32_t p = net_start[k]; p < net_start[k + 1]; ++p) {
        const int32_t c = pin_var[p];
        if (c < 0) continue;
        const float2 v = reinterpret_cast<const float2 *>(h + static_cast<int64_t>(c) * HID)[lane];
        a0 += v.x;
        a1 += v.y;
    }
    const float inv = net_mov[k] > 0 ? 1.0f / static_cast<float>(net_mov[k]) : 0.0f;
    reinterpret_cast<float2 *>(m + static_cast<int64_t>(k) * HID)[lane] = make_float2(a0 * inv, a1 * inv);
}

// g[c] = (1/cnt_c) sum over pins of cell c of e[net]
__global__ void k_nets_to_cells(const int32_t *pin_start, const int2 *pin_ref, int32_t n,
                                const float *e, float *g) {
    const int32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= n) return;
    float a0 = 0.f, a1 = 0.f;
    const int32_t e0 = pin_start[c], e1 = pin_start[c + 1];
    for (int32_t q = e0; q < e1; ++q) {
        const int32_t k = pin_ref[q].x;
        const float2 v = reinterpret_cast<const float2 *>(e + static_cast<int64_t>(k) * HID)[lane];
        a0 += v.x;
        a1 += v.y;
    }
    const float inv = e1 > e0 ? 1.0f / static_cast<float>(e1 - e0) : 0.0f;
    reinterpret_cast<float2 *>(g + static_cast<int64_t>(c) * HID)[lane] = make_float2(a0 * inv, a1 * inv);
}

// dh[c] (+)= sum over pins of cell c of dm[net] / cnt_net   (transpose of cells->nets)
__global__ void k_cells_to_nets_T(const int32_t *pin_start, const int2 *pin_ref,
                                  const int32_t *net_mov, int32_t n, const float *dm, float *dh,
                                  int accumulate) {
    const int32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= n) return;
    float a0 = 0.f, a1 = 0.f;
    for (int32_t q = pin_start[c]; q < pin_start[c + 1]; ++q) {
        const int32_t k = pin_ref[q].x;
        const float inv = 1.0f / static_cast<float>(net_mov[k]);
        const float2 v = reinterpret_cast<const float2 *>(dm + static_cast<int64_t>(k) * HID)[lane];
        a0 += v.x * inv;
        a1 += v.y * inv;
    }
    float2 *o = reinterpret_cast<float2 *>(dh + static_cast<int64_t>(c) * HID) + lane;
    if (accumulate) {
        const float2 old = *o;
        a0 += old.x;
        a1 += old.y;
    }
    *o = make_float2(a0, a1);
}

// de[k] = sum over movable pins of net k of dg[cell] / cnt_cell   (transpose of nets->cells)
__global__ void k_nets_to_cells_T(const int32_t *net_start, const int32_t *pin_var,
                                  const int32_t *pin_start, int32_t N, const float *dg, float *de) {
    const int32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (k >= N) return;
    float a0 = 0.f, a1 = 0.f;
    for (int32_t p = net_start[k]; p < net_start[k + 1]; ++p) {
        const int32_t c = pin_var[p];
        if (c < 0) continue;
        const float inv = 1.0f / static_cast<float>(pin_start[c + 1] - pin_start[c]);
        const float2 v = reinterpret_cast<const float2 *>(dg + static_cast<int64_t>(c) * HID)[lane];
        a0 += v.x * inv;
        a1 += v.y * inv;
    }
    reinterpret_cast<float2 *>(de + static_cast<int64_t>(k) * HID)[lane] = make_float2(a0, a1);
}

// ---------------------------------------------------------------------------
// dense layers: Y[R x OUT] = act(X1 W1 + X2 W2 + b), K in {8 (padded), 64}
// ---------------------------------------------------------------------------
struct DenseArgs {
    const float *x1;       // [R x K]
    const float *x2;       // [R x 64] or null
    const float *w1;       // FP32 [K x OUT] (or [OUT x K] when transposed)
    const float *w2;
    const __nv_bfloat16 *w1h;  // BF16 copies (tensor-core path)
    const __nv_bfloat16 *w2h;
    const float *bias;     // [OUT] or null
    const float *mask;     // [R x K]: when set, X1 is multiplied by (mask > 0)
    float *y;              // [R x OUT]
    int32_t rows;
    int32_t k;             // input width (8, 16 or 64)
    int32_t out;           // output width (16 or 64)
    int32_t relu;
    int32_t transpose;     // weights stored [OUT x K] (use W^T)
    int32_t accumulate;    // y += result
};

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&v);
}

// Tensor-core path: one warp per 16 rows; weights staged in shared memory as
// BF16 [K][OUT] (K padded to a multiple of 16).
template <int KMAX, int OUTMAX>
__global__ void __launch_bounds__(128) k_dense_tc(DenseArgs A) {
    __shared__ __nv_bfloat16 w1s[KMAX * OUTMAX];
    __shared__ __nv_bfloat16 w2s[64 * OUTMAX];
    const int kpad = (A.k + 15) & ~15;
    for (int idx = threadIdx.x; idx < kpad * A.out; idx += blockDim.x) {
        const int kk = idx / A.out, nn = idx % A.out;
        __nv_bfloat16 v = __float2bfloat16(0.0f);
        if (kk < A.k) v = A.transpose ? A.w1h[nn * A.k + kk] : A.w1h[kk * A.out + nn];
        w1s[kk * A.out + nn] = v;
    }
    if (A.x2)
        for (int idx = threadIdx.x; idx < 64 * A.out; idx += blockDim.x) {
            const int kk = idx / A.out, nn = idx % A.out;
            w2s[kk * A.out + nn] = A.transpose ? A.w2h[nn * 64 + kk] : A.w2h[kk * A.out + nn];
        }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int64_t r0 = (static_cast<int64_t>(blockIdx.x) * 4 + warp) * 16;
    if (r0 >= A.rows) return;
    const int ntiles = A.out / 8;
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
    auto xval = [&](const float *X, int width, int64_t row, int col, bool masked) -> float {
        if (row >= A.rows || col >= width) return 0.0f;
        float v = X[row * width + col];
        if (masked && !(A.mask[row * width + col] > 0.0f)) v = 0.0f;
        return v;
    };
    auto mma_pass = [&](const float *X, int width, const __nv_bfloat16 *ws, bool masked) {
        const int kp = (width + 15) & ~15;
        for (int k0 = 0; k0 < kp; k0 += 16) {
            uint32_t a[4];
            a[0] = pack_bf16(xval(X, width, r0 + g, k0 + 2 * t, masked),
                             xval(X, width, r0 + g, k0 + 2 * t + 1, masked));
            a[1] = pack_bf16(xval(X, width, r0 + g + 8, k0 + 2 * t, masked),
                             xval(X, width, r0 + g + 8, k0 + 2 * t + 1, masked));
            a[2] = pack_bf16(xval(X, width, r0 + g, k0 + 2 * t + 8, masked),
                             xval(X, width, r0 + g, k0 + 2 * t + 9, masked));
            a[3] = pack_bf16(xval(X, width, r0 + g + 8, k0 + 2 * t + 8, masked),
                             xval(X, width, r0 + g + 8, k0 + 2 * t + 9, masked));
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (j >= ntiles) break;
                const int nn = j * 8 + g;
                __nv_bfloat162 b0v, b1v;
                b0v.x = ws[(k0 + 2 * t) * A.out + nn];
                b0v.y = ws[(k0 + 2 * t + 1) * A.out + nn];
                b1v.x = ws[(k0 + 2 * t + 8) * A.out + nn];
                b1v.y = ws[(k0 + 2 * t + 9) * A.out + nn];
                const uint32_t b0 = *reinterpret_cast<uint32_t *>(&b0v);
                const uint32_t b1 = *reinterpret_cast<uint32_t *>(&b1v);
                asm volatile(
                    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                    "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                    : "+f"(acc[j][0]), "+f"(acc[j][1]), "+f"(acc[j][2]), "+f"(acc[j][3])
                    : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
            }
        }
    };
    mma_pass(A.x1, A.k, w1s, A.mask != nullptr);
    if (A.x2) mma_pass(A.x2, 64, w2s, false);
    for (int j = 0; j < ntiles; ++j) {
        const int c0 = j * 8 + 2 * t;
        const float b0 = A.bias ? A.bias[c0] : 0.0f;
        const float b1 = A.bias ? A.bias[c0 + 1] : 0.0f;
        const int64_t ra = r0 + g, rb = r0 + g + 8;
        float v[4] = {acc[j][0] + b0, acc[j][1] + b1, acc[j][2] + b0, acc[j][3] + b1};
        if (A.relu)
            for (int q = 0; q < 4; ++q) v[q] = v[q] > 0.0f ? v[q] : 0.0f;
        if (ra < A.rows) {
            float *o = A.y + ra * A.out + c0;
            if (A.accumulate) { v[0] += o[0]; v[1] += o[1]; }
            o[0] = v[0];
            o[1] = v[1];
        }
        if (rb < A.rows) {
            float *o = A.y + rb * A.out + c0;
            if (A.accumulate) { v[2] += o[0]; v[3] += o[1]; }
            o[0] = v[2];
            o[1] = v[3];
        }
    }
}

// ---------------------------------------------------------------------------
// The same layer on the 5th-generation tensor cores (tcgen05.mma, sm_100a).
//
// A persistent CTA of eight warps stages the weights once as the MMA's B
// operand (OUT x K, K-major, BF16) and then walks 128-row tiles: the threads
// convert the tile's rows of X1 (masked) and X2 to BF16 in shared memory (A
// operand, 128 x K, K-major), one thread issues K/16 tcgen05.mma (kind::f16,
// M = 128, N = OUT, FP32 accumulator in tensor memory) and commits them to an
// mbarrier, and warps w and w + 4 read accumulator lanes 32 w .. 32 w + 31
// (= rows), alternate 16-column chunks each, back with tcgen05.ld for the
// bias / ReLU / accumulate epilogue. K = kpad(K1) + 64 when
// X2 is present (at most 128), so one tile is at most eight MMAs.
// Operand layout (no swizzle, K-major): 8 x 8 core matrices of 16-byte rows;
// element (r, k) sits at (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 +
// (k % 8) * 2 bytes, SBO = (K / 8) * 128 (the descriptor's leading offset is
// the 128-byte step to the next 8 k, its stride offset SBO the step to the
// next 8 rows).
// ---------------------------------------------------------------------------
constexpr int kUmmaM = 128;
constexpr int kUmmaKMax = 128;
constexpr int kUmmaNMax = 64;
constexpr uint32_t kUmmaTmemCols = 64;  // power of two >= 32, >= OUT
constexpr int kUmmaSmemA = kUmmaM * kUmmaKMax * 2;     // 32 KiB
constexpr int kUmmaSmemB = kUmmaNMax * kUmmaKMax * 2;  // 16 KiB
// Eight warps per CTA and a grid of four CTAs per SM. Dynamic shared memory
// per CTA bounds how many CTAs can share an SM (228 KiB), and with it the
// tensor memory they hold (64 of the SM's 512 columns each), so that
// tcgen05.alloc never waits on another CTA: layers with K <= 64 take 26 KiB
// (at most eight CTAs, 8 x 64 columns), layers with K = 128 49 KiB (at most
// four).
constexpr int kUmmaThreads = 256;
constexpr int kUmmaSmem = kUmmaSmemA + kUmmaSmemB + 1024;
constexpr int kUmmaSmemSmall = 26 * 1024;
constexpr int kUmmaCtasPerSm = 4;
constexpr uint64_t kUmmaWaitNs = 200ull * 1000 * 1000;  // bound on one tile's MMA wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start, leading and stride byte offsets
// (each >> 4), descriptor version 1 (sm_100), no swizzle, base offset 0.
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) |
           (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16
// A and B (bits 7-9 and 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at
// bit 24.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(kUmmaM >> 4) << 24);
}

__device__ __forceinline__ uint32_t core_offset(int r, int k, int sbo) {
    return static_cast<uint32_t>((r >> 3) * sbo + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Bounded wait for an mbarrier phase; false when the bound ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
    const uint64_t t0 = ktg::global_timer_ns();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
        if (ktg::global_timer_ns() - t0 > limit_ns) return false;
    }
}

struct UmmaArgs {
    DenseArgs d;
    int *status;  // set to 1 when a tile's MMA wait ran out (the layer's output is then invalid)
};

__global__ void __launch_bounds__(kUmmaThreads, kUmmaCtasPerSm) k_dense_umma(UmmaArgs U) {
    const DenseArgs &A = U.d;
    extern __shared__ __align__(1024) uint8_t umma_smem[];
    uint8_t *sa = umma_smem;
    uint8_t *sb;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base_s;
    __shared__ float bias_s[kUmmaNMax];
    __shared__ int abort_s;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kp1 = (A.k + 15) & ~15;
    const int kt = kp1 + (A.x2 ? 64 : 0);
    const int sbo = (kt / 8) * 128;
    const int out = A.out;
    sb = sa + kUmmaM * kt * 2;  // B follows the 128 x K A tile

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_base_s)), "r"(kUmmaTmemCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_s = 0;
    }
    // B operand: B[n][k] = W1[k][n] for k < kp1 (zero past K1), W2[k - kp1][n] after
    for (int idx = threadIdx.x; idx < out * kt; idx += blockDim.x) {
        // consecutive threads read consecutive weights ([OUT x K] or [K x OUT])
        int nn, kk;
        if (A.transpose) {
            nn = idx / kt;
            kk = idx - nn * kt;
        } else {
            kk = idx / out;
            nn = idx - kk * out;
        }
        __nv_bfloat16 v = __float2bfloat16(0.0f);
        if (kk < kp1) {
            if (kk < A.k) v = A.transpose ? A.w1h[nn * A.k + kk] : A.w1h[kk * out + nn];
        } else {
            const int k2 = kk - kp1;
            v = A.transpose ? A.w2h[nn * 64 + k2] : A.w2h[k2 * out + nn];
        }
        *reinterpret_cast<__nv_bfloat16 *>(sb + core_offset(nn, kk, sbo)) = v;
    }
    for (int c = threadIdx.x; c < out; c += blockDim.x) bias_s[c] = A.bias ? A.bias[c] : 0.0f;

    const int64_t tiles = (static_cast<int64_t>(A.rows) + kUmmaM - 1) / kUmmaM;
    const int chunks = kt / 8;  // 16-byte rows of 8 k per operand row
    const uint32_t idesc = umma_idesc_bf16(out);
    uint32_t phase = 0;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int64_t row0 = tile * kUmmaM;
        // A operand: rows of X1 (masked, zero past K1) then X2, as BF16
        for (int idx = threadIdx.x; idx < kUmmaM * chunks; idx += blockDim.x) {
            const int r = idx / chunks, kc = idx - r * chunks;
            const int64_t row = row0 + r;
            float v[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
            if (row < A.rows) {
                const int k0 = kc * 8;
                if (k0 < kp1) {
                    if (k0 < A.k) {  // K1 is a multiple of 8: the chunk lies inside X1
                        const float4 *src = reinterpret_cast<const float4 *>(A.x1 + row * A.k + k0);
                        const float4 a = __ldg(src), b = __ldg(src + 1);
                        v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
                        v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
                        if (A.mask) {
                            const float4 *ms = reinterpret_cast<const float4 *>(A.mask + row * A.k + k0);
                            const float4 ma = __ldg(ms), mb = __ldg(ms + 1);
                            const float mv[8] = {ma.x, ma.y, ma.z, ma.w, mb.x, mb.y, mb.z, mb.w};
#pragma unroll
                            for (int q = 0; q < 8; ++q)
                                if (!(mv[q] > 0.0f)) v[q] = 0.0f;
                        }
                    }
                } else {
                    const float4 *src =
                        reinterpret_cast<const float4 *>(A.x2 + row * 64 + (k0 - kp1));
                    const float4 a = __ldg(src), b = __ldg(src + 1);
                    v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
                    v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
                }
            }
            uint4 pk;
            pk.x = pack_bf16(v[0], v[1]);
            pk.y = pack_bf16(v[2], v[3]);
            pk.z = pack_bf16(v[4], v[5]);
            pk.w = pack_bf16(v[6], v[7]);
            *reinterpret_cast<uint4 *>(sa + core_offset(r, kc * 8, sbo)) = pk;
        }
        // shared-memory writes -> visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        const uint32_t tmem = tmem_base_s;
        if (threadIdx.x == 0) {
            const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
            for (int ks = 0; ks < kt / 16; ++ks) {
                const uint64_t ad = umma_smem_desc(a0 + ks * 256, 128, sbo);
                const uint64_t bd = umma_smem_desc(b0 + ks * 256, 128, sbo);
                const uint32_t acc = ks > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    :: "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc) : "memory");
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                :: "r"(smem_u32(&mbar)) : "memory");
        }
        if (!mbar_wait_bounded(smem_u32(&mbar), phase, kUmmaWaitNs)) abort_s = 1;
        phase ^= 1u;
        tc_fence_after();
        __syncthreads();
        if (abort_s) break;
        // epilogue: warp w reads accumulator lanes 32 (w % 4) .. + 31 (its
        // rows); with eight warps, warps 4-7 take every other 16 columns
        const int quad = warp & 3;
        const int64_t row = row0 + quad * 32 + lane;
        const int cstep = 16 * static_cast<int>(blockDim.x >> 7);
        for (int c0 = 16 * (warp >> 2); c0 < out; c0 += cstep) {
            uint32_t rg[16];
            const uint32_t taddr = tmem + (static_cast<uint32_t>(quad * 32) << 16) + c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(rg[0]), "=r"(rg[1]), "=r"(rg[2]), "=r"(rg[3]), "=r"(rg[4]), "=r"(rg[5]),
                  "=r"(rg[6]), "=r"(rg[7]), "=r"(rg[8]), "=r"(rg[9]), "=r"(rg[10]), "=r"(rg[11]),
                  "=r"(rg[12]), "=r"(rg[13]), "=r"(rg[14]), "=r"(rg[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < A.rows) {
                float v[16];
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    v[q] = __uint_as_float(rg[q]) + bias_s[c0 + q];
                    if (A.relu) v[q] = v[q] > 0.0f ? v[q] : 0.0f;
                }
                float4 *dst = reinterpret_cast<float4 *>(A.y + row * out + c0);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    float4 o = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                    if (A.accumulate) {
                        const float4 p = dst[q];
                        o.x += p.x, o.y += p.y, o.z += p.z, o.w += p.w;
                    }
                    dst[q] = o;
                }
            }
        }
        // every warp's reads of the accumulator end before the next tile's MMA
        tc_fence_before();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (abort_s && threadIdx.x == 0) atomicExch(U.status, 1);
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem_base_s), "r"(kUmmaTmemCols) : "memory");
}

// FP32 CUDA-core path of the same operation (one thread per output element).
__global__ void k_dense_fp32(DenseArgs A) {
    const int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (idx >= static_cast<int64_t>(A.rows) * A.out) return;
    const int64_t r = idx / A.out;
    const int nn = static_cast<int>(idx % A.out);
    float s = A.bias ? A.bias[nn] : 0.0f;
    for (int kk = 0; kk < A.k; ++kk) {
        float xv = A.x1[r * A.k + kk];
        if (A.mask && !(A.mask[r * A.k + kk] > 0.0f)) xv = 0.0f;
        const float w = A.transpose ? A.w1[nn * A.k + kk] : A.w1[kk * A.out + nn];
        s += xv * w;
    }
    if (A.x2)
        for (int kk = 0; kk < 64; ++kk) {
            const float w = A.transpose ? A.w2[nn * 64 + kk] : A.w2[kk * A.out + nn];
            s += A.x2[r * 64 + kk] * w;
        }
    if (A.relu) s = s > 0.0f ? s : 0.0f;
    if (A.accumulate) s += A.y[idx];
    A.y[idx] = s;
}

// Weight gradient dW[K x OUT] = X^T (dY * mask) and db = sum rows of
// (dY * mask), per block over a strided set of 64-row chunks, written as
// block partials; k_reduce_partials sums blocks in order (deterministic).
__global__ void __launch_bounds__(256) k_wgrad(const float *x, int32_t k, const float *dy,
                                                const float *ymask, int32_t out, int32_t rows,
                                                float *partials) {
    __shared__ float xs[64 * 64];
    __shared__ float ds[64 * 64];
    const int nout = k * out + out;  // dW then db
    float acc[20];
#pragma unroll
    for (int q = 0; q < 20; ++q) acc[q] = 0.0f;
    for (int64_t c0 = static_cast<int64_t>(blockIdx.x) * 64; c0 < rows;
         c0 += static_cast<int64_t>(gridDim.x) * 64) {
        const int cr = rows - c0 < 64 ? static_cast<int>(rows - c0) : 64;
        for (int idx = threadIdx.x; idx < 64 * k; idx += blockDim.x) {
            const int rr = idx / k;
            xs[idx] = rr < cr ? x[(c0 + rr) * k + idx % k] : 0.0f;
        }
        for (int idx = threadIdx.x; idx < 64 * out; idx += blockDim.x) {
            const int rr = idx / out;
            float v = 0.0f;
            if (rr < cr) {
                const int64_t o = (c0 + rr) * out + idx % out;
                v = dy[o];
                if (ymask && !(ymask[o] > 0.0f)) v = 0.0f;
            }
            ds[idx] = v;
        }
        __syncthreads();
        for (int q = 0; q < 20; ++q) {
            const int oi = threadIdx.x + q * blockDim.x;
            if (oi >= nout) break;
            float s = 0.0f;
            if (oi < k * out) {
                const int a = oi / out, b = oi % out;
                for (int rr = 0; rr < 64; ++rr) s += xs[rr * k + a] * ds[rr * out + b];
            } else {
                const int b = oi - k * out;
                for (int rr = 0; rr < 64; ++rr) s += ds[rr * out + b];
            }
            acc[q] += s;
        }
        __syncthreads();
    }
    for (int q = 0; q < 20; ++q) {
        const int oi = threadIdx.x + q * blockDim.x;
        if (oi >= nout) break;
        partials[static_cast<int64_t>(blockIdx.x) * nout + oi] = acc[q];
    }
}

__global__ void k_reduce_partials(const float *partials, int blocks, int nout, float *dw,
                                  float *db, int kout) {
    const int oi = blockIdx.x * blockDim.x + threadIdx.x;
    if (oi >= nout) return;
    float s = 0.0f;
    for (int b = 0; b < blocks; ++b) s += partials[static_cast<int64_t>(b) * nout + oi];
    if (oi < kout)
        dw[oi] += s;
    else if (db)
        db[oi - kout] += s;
}

// ---------------------------------------------------------------------------
// learned coarse vector: topology features, head, projection loss
// ---------------------------------------------------------------------------
// Per-cell features of the netlist alone (no positions), the trunk's input
// when it predicts the coarse vector; computed once per netlist:
//   1, pins/8, mean over the cell's nets of (movable pins - 1)/8, of fixed
//   pins/4, share of its nets with a fixed pin, mean 1/(degree - 1),
//   log(area)/8, log1p(pins)/2.
__global__ void k_topo_features(const int32_t *pin_start, const int2 *pin_ref,
                                const int32_t *net_start, const int32_t *net_mov,
                                const double *area, int32_t n, float *x) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t e0 = pin_start[i], e1 = pin_start[i + 1];
    double smov = 0.0, sfix = 0.0, anyfix = 0.0, sinv = 0.0;
    for (int32_t q = e0; q < e1; ++q) {
        const int32_t k = pin_ref[q].x;
        const int32_t deg = net_start[k + 1] - net_start[k];
        const int32_t mov = net_mov[k];
        smov += mov - 1;
        sfix += deg - mov;
        anyfix += deg > mov ? 1.0 : 0.0;
        sinv += deg >= 2 ? 1.0 / (deg - 1) : 0.0;
    }
    const double k = static_cast<double>(e1 - e0);
    const double inv = k > 0.0 ? 1.0 / k : 0.0;
    const double a = area[i];
    float *xi = x + static_cast<int64_t>(i) * NFEAT;
    xi[0] = 1.0f;
    xi[1] = static_cast<float>(k / 8.0);
    xi[2] = static_cast<float>(smov * inv / 8.0);
    xi[3] = static_cast<float>(sfix * inv / 4.0);
    xi[4] = static_cast<float>(anyfix * inv);
    xi[5] = static_cast<float>(sinv * inv);
    xi[6] = static_cast<float>(a > 0.0 ? log(a) / 8.0 : 0.0);
    xi[7] = static_cast<float>(log1p(k) / 2.0);
}

struct HeadArgs {
    const int32_t *rp;
    const double *val;
    const double *diag;
    int32_t n;
    const double *logd_mean;
    const float *p;   // [n x PROJ] trunk embedding
    const float *w;   // parameters (FP32 master)
    int64_t Wh, bh, wz, bz;
    float *u;         // [n x HEAD_IN] head inputs (training) or null
    float *hh;        // [n x HEAD_H] hidden activations (training) or null
    float *o;         // [n] pre-softplus output (training) or null
    double *zd;       // [n] z in FP64 (training) or null
    float *zf;        // [n] z in FP32 (inference) or null
};

// z_i = softplus(relu(u_i Wh + bh) . wz + bz), u_i = (p_i, c_i, l_i) with the
// coupling share c_i = sum_j |a_ij| / a_ii and l_i = log a_ii - mean log a.
__global__ void __launch_bounds__(256) k_coarse_head(HeadArgs A) {
    __shared__ float ws[HEAD_IN * HEAD_H + 2 * HEAD_H + 1];
    for (int t = threadIdx.x; t < HEAD_IN * HEAD_H; t += blockDim.x) ws[t] = A.w[A.Wh + t];
    for (int t = threadIdx.x; t < HEAD_H; t += blockDim.x) {
        ws[HEAD_IN * HEAD_H + t] = A.w[A.bh + t];
        ws[HEAD_IN * HEAD_H + HEAD_H + t] = A.w[A.wz + t];
    }
    if (threadIdx.x == 0) ws[HEAD_IN * HEAD_H + 2 * HEAD_H] = A.w[A.bz];
    __syncthreads();
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    double rowabs = 0.0;
    for (int32_t e = A.rp[i]; e < A.rp[i + 1]; ++e) rowabs += fabs(A.val[e]);
    const double d = A.diag[i];
    float u[HEAD_IN];
#pragma unroll
    for (int k = 0; k < PROJ; ++k) u[k] = A.p[static_cast<int64_t>(i) * PROJ + k];
    u[PROJ] = static_cast<float>(rowabs / d);
    u[PROJ + 1] = static_cast<float>(log(d) - *A.logd_mean);
    float o = ws[HEAD_IN * HEAD_H + 2 * HEAD_H];
#pragma unroll
    for (int j = 0; j < HEAD_H; ++j) {
        float t = ws[HEAD_IN * HEAD_H + j];
#pragma unroll
        for (int k = 0; k < HEAD_IN; ++k) t += u[k] * ws[k * HEAD_H + j];
        t = t > 0.0f ? t : 0.0f;
        if (A.hh) A.hh[static_cast<int64_t>(i) * HEAD_H + j] = t;
        o += t * ws[HEAD_IN * HEAD_H + HEAD_H + j];
    }
    const float z = o > 20.0f ? o : log1pf(expf(o));
    if (A.u)
#pragma unroll
        for (int k = 0; k < HEAD_IN; ++k) A.u[static_cast<int64_t>(i) * HEAD_IN + k] = u[k];
    if (A.o) A.o[i] = o;
    if (A.zd) A.zd[i] = z;
    if (A.zf) A.zf[i] = z;
}

// out = A in (FP64, one thread per row; training only).
__global__ void k_spmv_rows(const int32_t *rp, const int32_t *col, const double *val,
                            const double *diag, int32_t n, const double *in, double *out) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = diag[i] * in[i];
    for (int32_t e = rp[i]; e < rp[i + 1]; ++e) s += val[e] * in[col[e]];
    out[i] = s;
}

// Projection loss of the test vectors e_t on z in the A-inner product,
//   L = (1/T) sum_t (1 - (z^T A e_t)^2 / ((z^T A z)(e_t^T A e_t))),
// from az = A z and a_t = A e_t: block partials of q = z.az, p_t = z.a_t,
// S_t = e_t.a_t, summed in block order by the last block, which writes
// out = {L, beta, alpha_0..alpha_{T-1}, q, p_0.., S_0..} with
// dL/dz = beta az + sum_t alpha_t a_t.
__global__ void __launch_bounds__(256) k_coarse_dots(int32_t n, int T, const double *z,
                                                     const double *az, const double *a,
                                                     const double *e, double *partials,
                                                     unsigned *ticket, double *out) {
    __shared__ double red[33 * (1 + 2 * kMaxVec)];
    constexpr int K = 1 + 2 * kMaxVec;
    double v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = 0.0;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double zi = z[i];
        v[0] += zi * az[i];
#pragma unroll
        for (int t = 0; t < kMaxVec; ++t) {
            if (t >= T) break;
            const double at = a[static_cast<int64_t>(t) * n + i];
            v[1 + t] += zi * at;
            v[1 + kMaxVec + t] += e[static_cast<int64_t>(t) * n + i] * at;
        }
    }
    block_sum_k<K>(v, red);
    if (threadIdx.x == 0)
        for (int k = 0; k < K; ++k) __stcg(partials + static_cast<int64_t>(blockIdx.x) * K + k, v[k]);
    if (last_block_done(ticket)) {
        double t[K];
#pragma unroll
        for (int k = 0; k < K; ++k) t[k] = 0.0;
        for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += blockDim.x)
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] += __ldcg(partials + static_cast<int64_t>(b) * K + k);
        block_sum_k<K>(t, red);
        if (threadIdx.x == 0) {
            const double q = t[0];
            double L = 0.0, beta = 0.0;
            int used = 0;
            for (int j = 0; j < T; ++j)
                if (t[1 + kMaxVec + j] > 0.0) ++used;
            for (int j = 0; j < T; ++j) {
                const double pj = t[1 + j], Sj = t[1 + kMaxVec + j];
                double al = 0.0;
                if (q > 0.0 && Sj > 0.0) {
                    L += (1.0 - pj * pj / (q * Sj)) / used;
                    al = -2.0 * pj / (used * q * Sj);
                    beta += 2.0 * pj * pj / (used * q * q * Sj);
                }
                out[2 + j] = al;
                out[2 + kMaxVec + 1 + j] = pj;
                out[2 + 2 * kMaxVec + 1 + j] = Sj;
            }
            out[0] = L;
            out[1] = beta;
            out[2 + kMaxVec] = q;
        }
    }
}

__global__ void k_coarse_dz(int32_t n, int T, const double *az, const double *a,
                            const double *coef, float *dz) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double g = coef[1] * az[i];
    for (int t = 0; t < T; ++t) g += coef[2 + t] * a[static_cast<int64_t>(t) * n + i];
    dz[i] = static_cast<float>(g);
}

// Head backward per row: d o = dz sigmoid(o); dh = d o wz (h > 0);
// du = dh Wh^T, whose first PROJ entries are dL/dp.
__global__ void __launch_bounds__(256) k_coarse_head_bwd(int32_t n, const float *w, int64_t Wh,
                                                         int64_t wz, const float *hh,
                                                         const float *o, const float *dz,
                                                         float *dhh, float *dout, float *dp) {
    __shared__ float ws[HEAD_IN * HEAD_H + HEAD_H];
    for (int t = threadIdx.x; t < HEAD_IN * HEAD_H; t += blockDim.x) ws[t] = w[Wh + t];
    for (int t = threadIdx.x; t < HEAD_H; t += blockDim.x) ws[HEAD_IN * HEAD_H + t] = w[wz + t];
    __syncthreads();
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float oi = o[i];
    const float dod = dz[i] * (oi > 20.0f ? 1.0f : 1.0f / (1.0f + expf(-oi)));
    dout[i] = dod;
    float dh[HEAD_H];
#pragma unroll
    for (int j = 0; j < HEAD_H; ++j) {
        const float hv = hh[static_cast<int64_t>(i) * HEAD_H + j];
        dh[j] = hv > 0.0f ? dod * ws[HEAD_IN * HEAD_H + j] : 0.0f;
        dhh[static_cast<int64_t>(i) * HEAD_H + j] = dh[j];
    }
#pragma unroll
    for (int k = 0; k < PROJ; ++k) {
        float s = 0.0f;
#pragma unroll
        for (int j = 0; j < HEAD_H; ++j) s += dh[j] * ws[k * HEAD_H + j];
        dp[static_cast<int64_t>(i) * PROJ + k] = s;
    }
}

// ---------------------------------------------------------------------------
// entry head, probe loss and their gradients
// ---------------------------------------------------------------------------
__device__ __forceinline__ int32_t row_of_entry(const int32_t *rp, int32_t n, int32_t e) {
    int32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const int32_t mid = (lo + hi + 1) >> 1;
        if (rp[mid] <= e) lo = mid; else hi = mid - 1;
    }
    return lo;
}

constexpr float kTMax = 0.999f;

// s_e = clamp(tanh(<p_i, p_j>/4)) |a_e| / sqrt(d_i d_j); also stores t_e.
__global__ void k_head(const int32_t *rp, const int32_t *col, const double *val,
                       const double *diag, int32_t n, int32_t m, const float *p, float *t_out,
                       float *s_out) {
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const int32_t i = row_of_entry(rp, n, e);
    const int32_t j = col[e];
    const float4 *pi = reinterpret_cast<const float4 *>(p + static_cast<int64_t>(i) * PROJ);
    const float4 *pj = reinterpret_cast<const float4 *>(p + static_cast<int64_t>(j) * PROJ);
    float phi = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 a = pi[q], b = pj[q];
        phi += a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
    }
    const float th = tanhf(phi * 0.25f);
    const float t = fminf(fmaxf(th, -kTMax), kTMax);
    const float c = static_cast<float>(fabs(val[e]) / sqrt(diag[i] * diag[j]));
    // t_out keeps tanh itself (its clamped slope is zero past the bound)
    if (t_out) t_out[e] = th;
    s_out[e] = t * c;
}

// index of the entry (j, i) paired with each entry (i, j): the k-th copy of
// column j in row i pairs with the k-th copy of column i in row j (-1 when
// the pattern is not symmetric).
__global__ void k_transpose_index(const int32_t *rp, const int32_t *col, int32_t n, int32_t m,
                                  int32_t *tr) {
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const int32_t i = row_of_entry(rp, n, e);
    const int32_t j = col[e];
    int32_t k = 0;
    for (int32_t q = rp[i]; q < e; ++q) k += col[q] == j;
    int32_t found = -1;
    for (int32_t q = rp[j]; q < rp[j + 1]; ++q)
        if (col[q] == i) {
            if (k == 0) { found = q; break; }
            --k;
        }
    tr[e] = found;
}

__device__ __forceinline__ double probe_value(uint64_t seed, int j, int64_t i) {
    uint64_t h = static_cast<uint64_t>(i) * 0x9E3779B97F4A7C15ull;
    h ^= seed * 0x632BE59BD9B4E019ull + static_cast<uint64_t>(j) * 0xD1B54A32D192ED03ull;
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    return ((h >> 17) & 1ull) ? 1.0 : -1.0;
}

// u = A v for probe j (FP64)
__global__ void k_probe_spmv(const int32_t *rp, const int32_t *col, const double *val,
                             const double *diag, int32_t n, uint64_t seed, int j, double *u) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = diag[i] * probe_value(seed, j, i);
    for (int32_t e = rp[i]; e < rp[i + 1]; ++e) s += val[e] * probe_value(seed, j, col[e]);
    u[i] = s;
}

// q = u/d + dis * S (dis * u); gq = 2 (q - v) / (K n); loss partials.
__global__ void k_probe_loss(const int32_t *rp, const int32_t *col, const double *diag,
                             const float *sval, int32_t n, uint64_t seed, int j, int K,
                             const double *u, double *gq, double *partials, unsigned *ticket,
                             double *loss_acc) {
    __shared__ double scratch[40];
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double term = 0.0;
    if (i < n) {
        const double dis_i = 1.0 / sqrt(diag[i]);
        double su = 0.0;
        for (int32_t e = rp[i]; e < rp[i + 1]; ++e) {
            const int32_t c = col[e];
            su += static_cast<double>(sval[e]) * (u[c] / sqrt(diag[c]));
        }
        const double q = u[i] / diag[i] + dis_i * su;
        const double err = q - probe_value(seed, j, i);
        const double scale = 1.0 / (static_cast<double>(K) * n);
        gq[i] = 2.0 * err * scale;
        term = err * err * scale;
    }
    const double bs = block_sum(term, scratch);
    if (threadIdx.x == 0) __stcg(partials + blockIdx.x, bs);
    if (last_block_done(ticket)) {
        const double t = sum_partials(partials, gridDim.x, scratch);
        if (threadIdx.x == 0) *loss_acc += t;
    }
}

// ds_e += gq_i dis_i dis_j u_j
__global__ void k_probe_ds(const int32_t *rp, const int32_t *col, const double *diag, int32_t n,
                           int32_t m, const double *gq, const double *u, float *ds, int first) {
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const int32_t i = row_of_entry(rp, n, e);
    const int32_t j = col[e];
    const double v = gq[i] * u[j] / sqrt(diag[i] * diag[j]);
    ds[e] = first ? static_cast<float>(v) : ds[e] + static_cast<float>(v);
}

// dphi_e = ds_e c_e dt/dphi, with dt/dphi = 1 - tanh^2 inside the clamp, 0 outside
__global__ void k_dphi(const int32_t *rp, const int32_t *col, const double *val,
                       const double *diag, int32_t n, int32_t m, const float *t, const float *ds,
                       float *dphi) {
    const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const int32_t i = row_of_entry(rp, n, e);
    const int32_t j = col[e];
    const float c = static_cast<float>(fabs(val[e]) / sqrt(diag[i] * diag[j]));
    const float th = t[e];
    dphi[e] = fabsf(th) < kTMax ? ds[e] * c * (1.0f - th * th) : 0.0f;
}

// dp_i = sum over entries e=(i,j) of (dphi_e + dphi_tr(e)) p_j / 4
__global__ void k_dp(const int32_t *rp, const int32_t *col, const int32_t *tr, int32_t n,
                     const float *dphi, const float *p, float *dp) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float acc[PROJ];
#pragma unroll
    for (int q = 0; q < PROJ; ++q) acc[q] = 0.0f;
    for (int32_t e = rp[i]; e < rp[i + 1]; ++e) {
        const int32_t j = col[e];
        const float w = (dphi[e] + (tr[e] >= 0 ? dphi[tr[e]] : 0.0f)) * 0.25f;
        const float *pj = p + static_cast<int64_t>(j) * PROJ;
#pragma unroll
        for (int q = 0; q < PROJ; ++q) acc[q] += w * pj[q];
    }
#pragma unroll
    for (int q = 0; q < PROJ; ++q) dp[static_cast<int64_t>(i) * PROJ + q] = acc[q];
}

__global__ void k_to_bf16(const float *a, __nv_bfloat16 *b, int64_t n) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16(a[i]);
}

__global__ void k_adam(float *w, const float *g, float *m1, float *m2, int64_t n, float lr,
                       float b1, float b2, float eps, float c1, float c2, float clip_scale) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] * clip_scale;
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

__global__ void k_sumsq(const float *g, int64_t n, double *partials, unsigned *ticket,
                        double *out) {
    __shared__ double scratch[40];
    double v = 0.0;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        v += static_cast<double>(g[i]) * g[i];
    const double bs = block_sum(v, scratch);
    if (threadIdx.x == 0) __stcg(partials + blockIdx.x, bs);
    if (last_block_done(ticket)) {
        const double t = sum_partials(partials, gridDim.x, scratch);
        if (threadIdx.x == 0) *out = t;
    }
}

}  // namespace learned
}  // namespace ktg

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using namespace ktg::learned;

struct ktg_learned {
    int device = 0;
    std::string err;
    Layout L = layout();
    float *w = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    __nv_bfloat16 *wh = nullptr;
    int64_t step = 0;
    // dense layers: 2 tcgen05 (BF16 operands in shared memory, FP32
    // accumulator in tensor memory), 1 BF16 mma.sync, 0 FP32 CUDA cores
    int tensor_cores = 2;
    int num_sms = 148;
    int tc_ctas = 0;           // cap on the tcgen05 layers' persistent CTAs (0: 4 per SM)
    int *tc_status = nullptr;  // set by a tcgen05 layer whose MMA wait ran out
    bool umma_used = false;
    float lr = 1e-3f;
    int probes = 4;
    float clip = 1.0f;
    // work buffers (grown on demand)
    int64_t cap_rows = 0, cap_nets = 0, cap_nnz = 0;
    float *x = nullptr;                 // [n x 8]
    float *act_c = nullptr;             // cell activations: h0..h3, g0..g2 [7][n x 64]
    float *act_n = nullptr;             // net activations: m0..m2, e0..e2 [6][N x 64]
    float *p = nullptr, *dp = nullptr;  // [n x 16]
    float *dh = nullptr, *dh2 = nullptr, *dg = nullptr;  // [n x 64]
    float *dm = nullptr, *de = nullptr;                  // [N x 64]
    float *t = nullptr, *ds = nullptr, *dphi = nullptr;  // [m]
    int32_t *tr = nullptr;                               // [m]
    double *u = nullptr, *gq = nullptr;                  // [n]
    float *wpart = nullptr;                              // weight-gradient partials
    double *dpart = nullptr;                             // reduction partials
    unsigned *ticket = nullptr;
    double *scal = nullptr;                              // [4] logd mean, loss, gnorm
    double *h_scal = nullptr;
    cudaStream_t stream = nullptr;
    int64_t launches = 0;
    int64_t version = 0;  // bumped whenever the parameters change
    // coarse-vector network: work buffers (grown on demand)
    int64_t cap_coarse = 0;
    int cap_vec = 0;
    float *cu = nullptr, *chh = nullptr, *co = nullptr, *cdz = nullptr, *cdhh = nullptr,
          *cdo = nullptr;                                // [n x 18], [n x 16], [n] ...
    double *czd = nullptr, *caz = nullptr;               // [n]
    double *ce = nullptr, *ca = nullptr;                 // [T x n] test vectors, A e
    double *cscal = nullptr;                             // [2 + 3 * kMaxVec + 1]
    uint64_t uid = 0;  // process-unique id (tags the embeddings it leaves in contexts)
};

namespace {

constexpr int kWgradBlocks = 256;

int lerr(ktg_learned *h, int code, const std::string &m) {
    if (h) h->err = m;
    return code;
}

#define KTG_LCUDA(h, call)                                                                  \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return lerr((h), KTG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
int lalloc(ktg_learned *h, T **p, int64_t count) {
    if (*p) cudaFree(*p);
    *p = nullptr;
    KTG_LCUDA(h, cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * std::max<int64_t>(count, 1)));
    return KTG_OK;
}

int reserve_work(ktg_learned *h, int64_t n, int64_t N, int64_t m) {
    int rc;
    if (n > h->cap_rows) {
        const int64_t c = std::max(n, h->cap_rows * 3 / 2);
        if ((rc = lalloc(h, &h->x, c * NFEAT)) || (rc = lalloc(h, &h->act_c, 7 * c * HID)) ||
            (rc = lalloc(h, &h->p, c * PROJ)) || (rc = lalloc(h, &h->dp, c * PROJ)) ||
            (rc = lalloc(h, &h->dh, c * HID)) || (rc = lalloc(h, &h->dh2, c * HID)) ||
            (rc = lalloc(h, &h->dg, c * HID)) || (rc = lalloc(h, &h->u, c)) ||
            (rc = lalloc(h, &h->gq, c)))
            return rc;
        h->cap_rows = c;
    }
    if (N > h->cap_nets) {
        const int64_t c = std::max(N, h->cap_nets * 3 / 2);
        if ((rc = lalloc(h, &h->act_n, 6 * c * HID)) || (rc = lalloc(h, &h->dm, c * HID)) ||
            (rc = lalloc(h, &h->de, c * HID)))
            return rc;
        h->cap_nets = c;
    }
    if (m > h->cap_nnz) {
        const int64_t c = std::max(m, h->cap_nnz * 3 / 2);
        if ((rc = lalloc(h, &h->t, c)) || (rc = lalloc(h, &h->ds, c)) ||
            (rc = lalloc(h, &h->dphi, c)) || (rc = lalloc(h, &h->tr, c)))
            return rc;
        h->cap_nnz = c;
    }
    return KTG_OK;
}

struct SysView {
    const int32_t *rp;
    const int32_t *col;
    const double *val;
    const double *diag;
    int32_t n;
    int32_t m;
};

int sys_view(ktg_learned *h, ktg_ctx *c, int axis, SysView *v) {
    if (!c->have_netlist || !c->axis_valid[axis] || c->sys_n != c->n)
        return lerr(h, KTG_ERR_STATE, "context needs a B2B system of its netlist");
    int32_t m = 0;
    KTG_LCUDA(h, cudaMemcpy(&m, c->sys[axis].row_ptr + c->n, sizeof(int32_t), cudaMemcpyDeviceToHost));
    *v = SysView{c->sys[axis].row_ptr, c->sys[axis].col, c->sys[axis].val, c->sys[axis].diag,
                 static_cast<int32_t>(c->n), m};
    return KTG_OK;
}

float *cell_act(ktg_learned *h, int which) { return h->act_c + which * h->cap_rows * HID; }
float *net_act(ktg_learned *h, int which) { return h->act_n + which * h->cap_nets * HID; }
// cell activations: 0..3 = h0..h3, 4..6 = g0..g2; net activations: 0..2 = m, 3..5 = e

int dense(ktg_learned *h, const float *x1, int k, const float *x2, int64_t w1, int64_t w2,
          int64_t bias, float *y, int64_t rows, int out, bool relu, bool transpose,
          bool accumulate, const float *mask) {
    if (rows <= 0) return KTG_OK;
    ktg::learned::DenseArgs A;
    A.x1 = x1;
    A.x2 = x2;
    A.w1 = h->w + w1;
    A.w2 = x2 ? h->w + w2 : nullptr;
    A.w1h = h->wh + w1;
    A.w2h = x2 ? h->wh + w2 : nullptr;
    A.bias = bias >= 0 ? h->w + bias : nullptr;
    A.mask = mask;
    A.y = y;
    A.rows = static_cast<int32_t>(rows);
    A.k = k;
    A.out = out;
    A.relu = relu;
    A.transpose = transpose;
    A.accumulate = accumulate;
    auto aligned16 = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
    const bool umma_ok = h->tensor_cores == 2 && k % 8 == 0 && k <= 64 && out % 16 == 0 &&
                         out <= ktg::learned::kUmmaNMax && aligned16(x1) && aligned16(y) &&
                         (!x2 || aligned16(x2)) && (!mask || aligned16(mask));
    if (umma_ok) {
        const int64_t tiles = (rows + ktg::learned::kUmmaM - 1) / ktg::learned::kUmmaM;
        const int kt = ((k + 15) & ~15) + (x2 ? 64 : 0);
        const bool small = ktg::learned::kUmmaM * kt * 2 + out * kt * 2 <= ktg::learned::kUmmaSmemSmall;
        const int smem = small ? ktg::learned::kUmmaSmemSmall : ktg::learned::kUmmaSmem;
        int64_t cap = static_cast<int64_t>(h->num_sms) * ktg::learned::kUmmaCtasPerSm;
        if (h->tc_ctas > 0) cap = std::min<int64_t>(cap, h->tc_ctas);
        const int blocks = static_cast<int>(std::min<int64_t>(tiles, cap));
        ktg::learned::UmmaArgs U{A, h->tc_status};
        ktg::learned::k_dense_umma<<<blocks, ktg::learned::kUmmaThreads, smem, h->stream>>>(U);
        h->umma_used = true;
    } else if (h->tensor_cores) {
        const int blocks = static_cast<int>((rows + 63) / 64);
        ktg::learned::k_dense_tc<64, 64><<<blocks, 128, 0, h->stream>>>(A);
    } else {
        const int64_t total = rows * out;
        ktg::learned::k_dense_fp32<<<static_cast<int>((total + 255) / 256), 256, 0, h->stream>>>(A);
    }
    ++h->launches;
    KTG_LCUDA(h, cudaGetLastError());
    return KTG_OK;
}

int wgrad(ktg_learned *h, const float *x, int k, const float *dy, const float *ymask, int out,
          int64_t rows, int64_t wofs, int64_t bofs) {
    if (rows <= 0) return KTG_OK;
    const int nout = k * out + out;
    const int blocks = static_cast<int>(std::min<int64_t>(kWgradBlocks, (rows + 63) / 64));
    ktg::learned::k_wgrad<<<blocks, 256, 0, h->stream>>>(x, k, dy, ymask, out,
                                                         static_cast<int32_t>(rows), h->wpart);
    ktg::learned::k_reduce_partials<<<(nout + 255) / 256, 256, 0, h->stream>>>(
        h->wpart, blocks, nout, h->g + wofs, bofs >= 0 ? h->g + bofs : nullptr, k * out);
    h->launches += 2;
    KTG_LCUDA(h, cudaGetLastError());
    return KTG_OK;
}

// The trunk (message passing over the cell-net graph) from the features in
// h->x to the embedding p = h3 P in h->p.
// Reads the status word of the tcgen05 layers launched since the last check
// (one stream synchronisation; nothing when none ran).
int tc_check(ktg_learned *h) {
    if (!h->umma_used) return KTG_OK;
    h->umma_used = false;
    int st = 0;
    KTG_LCUDA(h, cudaMemcpyAsync(&st, h->tc_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    KTG_LCUDA(h, cudaStreamSynchronize(h->stream));
    if (st != 0) {
        cudaMemsetAsync(h->tc_status, 0, sizeof(int), h->stream);
        return lerr(h, KTG_ERR_TIMEOUT, "tensor-core dense layer: MMA completion wait ran out");
    }
    return KTG_OK;
}

int trunk_forward(ktg_learned *h, ktg_ctx *c, int64_t n) {
    int rc;
    const int64_t N = c->N;
    const Layout &L = h->L;
    if ((rc = dense(h, h->x, NFEAT, nullptr, L.W_in, 0, L.b_in, cell_act(h, 0), n, HID, true,
                    false, false, nullptr)))
        return rc;
    const int wpb = 8;  // warps per block for the aggregations
    for (int l = 0; l < LAYERS; ++l) {
        ktg::learned::k_cells_to_nets<<<static_cast<int>((N + wpb - 1) / wpb), 32 * wpb, 0, h->stream>>>(
            c->net_start, c->pin_var, c->net_mov, static_cast<int32_t>(N), cell_act(h, l),
            net_act(h, l));
        if ((rc = dense(h, net_act(h, l), HID, nullptr, L.Wa[l], 0, L.ba[l], net_act(h, 3 + l), N,
                        HID, true, false, false, nullptr)))
            return rc;
        ktg::learned::k_nets_to_cells<<<static_cast<int>((n + wpb - 1) / wpb), 32 * wpb, 0, h->stream>>>(
            c->pin_start, c->pin_ref, static_cast<int32_t>(n), net_act(h, 3 + l), cell_act(h, 4 + l));
        if ((rc = dense(h, cell_act(h, l), HID, cell_act(h, 4 + l), L.Wb[l], L.Wc[l], L.bb[l],
                        cell_act(h, l + 1), n, HID, true, false, false, nullptr)))
            return rc;
        h->launches += 2;
    }
    if ((rc = dense(h, cell_act(h, LAYERS), HID, nullptr, L.P, 0, -1, h->p, n, PROJ, false, false,
                    false, nullptr)))
        return rc;
    KTG_LCUDA(h, cudaGetLastError());
    return tc_check(h);
}

// Forward pass to p and the entry values (t, s) of one axis system (the
// learned sparse approximate inverse, system features as the trunk's input).
int forward(ktg_learned *h, ktg_ctx *c, const SysView &S, float *s_out, bool keep_t) {
    int rc;
    const int64_t n = S.n, N = c->N;
    if ((rc = reserve_work(h, n, N, S.m))) return rc;
    const int tb = 256;
    ktg::learned::k_logd_sum<<<std::min<int>(1024, (S.n + tb - 1) / tb + 1), tb, 0, h->stream>>>(
        S.diag, S.n, h->dpart, h->ticket, h->scal + 0);
    ktg::learned::k_features<<<(S.n + tb - 1) / tb, tb, 0, h->stream>>>(
        S.rp, S.col, S.val, S.diag, c->pin_start, S.n, h->scal + 0, h->x);
    h->launches += 2;
    if ((rc = trunk_forward(h, c, n))) return rc;
    if (S.m > 0) {
        ktg::learned::k_head<<<(S.m + tb - 1) / tb, tb, 0, h->stream>>>(
            S.rp, S.col, S.val, S.diag, S.n, S.m, h->p, keep_t ? h->t : nullptr, s_out);
        ++h->launches;
    }
    KTG_LCUDA(h, cudaGetLastError());
    return KTG_OK;
}

int trunk_backward(ktg_learned *h, ktg_ctx *c, int64_t n);

// Loss and gradients (accumulated into h->g, which the caller zeroes).
int loss_grad(ktg_learned *h, ktg_ctx *c, int axis, uint64_t seed, double *loss) {
    SysView S;
    int rc = sys_view(h, c, axis, &S);
    if (rc) return rc;
    if ((rc = reserve_work(h, S.n, c->N, S.m))) return rc;
    float *sval = h->dphi;  // reuse: s values, overwritten by dphi later
    if ((rc = forward(h, c, S, sval, true))) return rc;
    const int tb = 256;
    const int nblk = (S.n + tb - 1) / tb, mblk = (S.m + tb - 1) / tb;
    KTG_LCUDA(h, cudaMemsetAsync(h->scal + 1, 0, sizeof(double), h->stream));
    for (int j = 0; j < h->probes; ++j) {
        ktg::learned::k_probe_spmv<<<nblk, tb, 0, h->stream>>>(S.rp, S.col, S.val, S.diag, S.n,
                                                               seed, j, h->u);
        ktg::learned::k_probe_loss<<<nblk, tb, 0, h->stream>>>(
            S.rp, S.col, S.diag, sval, S.n, seed, j, h->probes, h->u, h->gq, h->dpart, h->ticket,
            h->scal + 1);
        if (S.m > 0)
            ktg::learned::k_probe_ds<<<mblk, tb, 0, h->stream>>>(S.rp, S.col, S.diag, S.n, S.m,
                                                                 h->gq, h->u, h->ds, j == 0);
        h->launches += 3;
    }
    if (S.m > 0) {
        ktg::learned::k_transpose_index<<<mblk, tb, 0, h->stream>>>(S.rp, S.col, S.n, S.m, h->tr);
        ktg::learned::k_dphi<<<mblk, tb, 0, h->stream>>>(S.rp, S.col, S.val, S.diag, S.n, S.m,
                                                         h->t, h->ds, h->dphi);
        h->launches += 2;
    }
    ktg::learned::k_dp<<<nblk, tb, 0, h->stream>>>(S.rp, S.col, h->tr, S.n, h->dphi, h->p, h->dp);
    ++h->launches;
    if ((rc = trunk_backward(h, c, S.n))) return rc;
    double l = 0.0;
    KTG_LCUDA(h, cudaMemcpyAsync(h->h_scal, h->scal + 1, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    KTG_LCUDA(h, cudaStreamSynchronize(h->stream));
    l = h->h_scal[0];
    if (loss) *loss = l;
    return tc_check(h);
}

// Gradients of the trunk's parameters from dL/dp in h->dp (accumulated into
// h->g), through the activations the last trunk_forward kept.
int trunk_backward(ktg_learned *h, ktg_ctx *c, int64_t n) {
    int rc;
    const Layout &L = h->L;
    const int64_t N = c->N;
    // p = h3 P: dP = h3^T dp, dh = dp P^T
    if ((rc = wgrad(h, cell_act(h, LAYERS), HID, h->dp, nullptr, PROJ, n, L.P, -1))) return rc;
    if ((rc = dense(h, h->dp, PROJ, nullptr, L.P, 0, -1, h->dh, n, HID, false, true, false, nullptr)))
        return rc;
    const int wpb = 8;
    for (int l = LAYERS - 1; l >= 0; --l) {
        // h_{l+1} = relu(h_l Wb + g_l Wc + bb): dz = dh * (h_{l+1} > 0)
        const float *hout = cell_act(h, l + 1);
        if ((rc = wgrad(h, cell_act(h, l), HID, h->dh, hout, HID, n, L.Wb[l], L.bb[l]))) return rc;
        if ((rc = wgrad(h, cell_act(h, 4 + l), HID, h->dh, hout, HID, n, L.Wc[l], -1))) return rc;
        // dh_prev = dz Wb^T ; dg = dz Wc^T   (dz = dh masked by hout)
        if ((rc = dense(h, h->dh, HID, nullptr, L.Wb[l], 0, -1, h->dh2, n, HID, false, true, false,
                        hout)))
            return rc;
        if ((rc = dense(h, h->dh, HID, nullptr, L.Wc[l], 0, -1, h->dg, n, HID, false, true, false,
                        hout)))
            return rc;
        // g = mean nets->cells (e): de = T(dg)
        ktg::learned::k_nets_to_cells_T<<<static_cast<int>((N + wpb - 1) / wpb), 32 * wpb, 0, h->stream>>>(
            c->net_start, c->pin_var, c->pin_start, static_cast<int32_t>(N), h->dg, h->de);
        ++h->launches;
        // e = relu(m Wa + ba): dza = de * (e > 0)
        const float *eout = net_act(h, 3 + l);
        if ((rc = wgrad(h, net_act(h, l), HID, h->de, eout, HID, N, L.Wa[l], L.ba[l]))) return rc;
        if ((rc = dense(h, h->de, HID, nullptr, L.Wa[l], 0, -1, h->dm, N, HID, false, true, false,
                        eout)))
            return rc;
        // m = mean cells->nets (h_l): dh_prev += T(dm)
        ktg::learned::k_cells_to_nets_T<<<static_cast<int>((n + wpb - 1) / wpb), 32 * wpb, 0, h->stream>>>(
            c->pin_start, c->pin_ref, c->net_mov, static_cast<int32_t>(n), h->dm, h->dh2, 1);
        ++h->launches;
        std::swap(h->dh, h->dh2);
    }
    // h0 = relu(x W_in + b_in)
    if ((rc = wgrad(h, h->x, NFEAT, h->dh, cell_act(h, 0), HID, n, L.W_in, L.b_in))) return rc;
    return KTG_OK;
}

int refresh_bf16(ktg_learned *h) {
    ktg::learned::k_to_bf16<<<static_cast<int>((h->L.total + 255) / 256), 256, 0, h->stream>>>(
        h->w, h->wh, h->L.total);
    ++h->launches;
    ++h->version;
    KTG_LCUDA(h, cudaGetLastError());
    return KTG_OK;
}

// ---- learned coarse vector ----------------------------------------------------

int reserve_coarse(ktg_learned *h, int64_t n, int T) {
    int rc;
    if (n > h->cap_coarse) {
        const int64_t c = std::max(n, h->cap_coarse * 3 / 2);
        if ((rc = lalloc(h, &h->cu, c * HEAD_IN)) || (rc = lalloc(h, &h->chh, c * HEAD_H)) ||
            (rc = lalloc(h, &h->co, c)) || (rc = lalloc(h, &h->cdz, c)) ||
            (rc = lalloc(h, &h->cdhh, c * HEAD_H)) || (rc = lalloc(h, &h->cdo, c)) ||
            (rc = lalloc(h, &h->czd, c)) || (rc = lalloc(h, &h->caz, c)))
            return rc;
        h->cap_coarse = c;
        h->cap_vec = 0;
    }
    if (T > h->cap_vec) {
        if ((rc = lalloc(h, &h->ce, h->cap_coarse * kMaxVec)) ||
            (rc = lalloc(h, &h->ca, h->cap_coarse * kMaxVec)))
            return rc;
        h->cap_vec = kMaxVec;
    }
    if (!h->cscal && (rc = lalloc(h, &h->cscal, 4 + 3 * kMaxVec))) return rc;
    return KTG_OK;
}

// The trunk on the netlist's topology features: h->p = embedding per cell.
int topo_trunk(ktg_learned *h, ktg_ctx *c) {
    const int64_t n = c->n;
    int rc;
    if ((rc = reserve_work(h, n, c->N, 0))) return rc;
    if (n > 0) {
        ktg::learned::k_topo_features<<<static_cast<int>((n + 255) / 256), 256, 0, h->stream>>>(
            c->pin_start, c->pin_ref, c->net_start, c->net_mov, c->area,
            static_cast<int32_t>(n), h->x);
        ++h->launches;
    }
    return trunk_forward(h, c, n);
}

HeadArgs head_args(ktg_learned *h, const SysView &S, const float *p) {
    HeadArgs A{};
    A.rp = S.rp;
    A.val = S.val;
    A.diag = S.diag;
    A.n = S.n;
    A.logd_mean = h->scal + 0;
    A.p = p;
    A.w = h->w;
    A.Wh = h->L.Wh;
    A.bh = h->L.bh;
    A.wz = h->L.wz;
    A.bz = h->L.bz;
    return A;
}

int logd_mean(ktg_learned *h, const SysView &S) {
    const int tb = 256;
    ktg::learned::k_logd_sum<<<std::min<int>(1024, (S.n + tb - 1) / tb + 1), tb, 0, h->stream>>>(
        S.diag, S.n, h->dpart, h->ticket, h->scal + 0);
    ++h->launches;
    KTG_LCUDA(h, cudaGetLastError());
    return KTG_OK;
}

// Projection loss of the host test vectors e [T x n] on the predicted z of
// one axis and its gradient (accumulated into h->g).
int coarse_loss_grad(ktg_learned *h, ktg_ctx *c, int axis, const double *e, int T,
                     double *loss) {
    SysView S;
    int rc = sys_view(h, c, axis, &S);
    if (rc) return rc;
    const int64_t n = S.n;
    if ((rc = reserve_coarse(h, n, T))) return rc;
    if ((rc = topo_trunk(h, c))) return rc;
    if ((rc = logd_mean(h, S))) return rc;
    const int tb = 256, nb = static_cast<int>((n + tb - 1) / tb);
    HeadArgs A = head_args(h, S, h->p);
    A.u = h->cu;
    A.hh = h->chh;
    A.o = h->co;
    A.zd = h->czd;
    ktg::learned::k_coarse_head<<<nb, tb, 0, h->stream>>>(A);
    KTG_LCUDA(h, cudaMemcpyAsync(h->ce, e, sizeof(double) * n * T, cudaMemcpyHostToDevice,
                                 h->stream));
    for (int t = 0; t < T; ++t)
        ktg::learned::k_spmv_rows<<<nb, tb, 0, h->stream>>>(S.rp, S.col, S.val, S.diag, S.n,
                                                            h->ce + t * n, h->ca + t * n);
    ktg::learned::k_spmv_rows<<<nb, tb, 0, h->stream>>>(S.rp, S.col, S.val, S.diag, S.n, h->czd,
                                                        h->caz);
    ktg::learned::k_coarse_dots<<<std::min(nb, 512), tb, 0, h->stream>>>(
        S.n, T, h->czd, h->caz, h->ca, h->ce, h->dpart, h->ticket, h->cscal);
    ktg::learned::k_coarse_dz<<<nb, tb, 0, h->stream>>>(S.n, T, h->caz, h->ca, h->cscal, h->cdz);
    ktg::learned::k_coarse_head_bwd<<<nb, tb, 0, h->stream>>>(
        S.n, h->w, h->L.Wh, h->L.wz, h->chh, h->co, h->cdz, h->cdhh, h->cdo, h->dp);
    h->launches += 5 + T;
    const Layout &L = h->L;
    if ((rc = wgrad(h, h->cu, HEAD_IN, h->cdhh, nullptr, HEAD_H, n, L.Wh, L.bh))) return rc;
    if ((rc = wgrad(h, h->chh, HEAD_H, h->cdo, nullptr, 1, n, L.wz, L.bz))) return rc;
    if ((rc = trunk_backward(h, c, n))) return rc;
    KTG_LCUDA(h, cudaMemcpyAsync(h->h_scal, h->cscal, sizeof(double), cudaMemcpyDeviceToHost,
                                 h->stream));
    KTG_LCUDA(h, cudaStreamSynchronize(h->stream));
    if (loss) *loss = h->h_scal[0];
    return KTG_OK;
}

int adam_step(ktg_learned *h) {
    ktg::learned::k_sumsq<<<64, 256, 0, h->stream>>>(h->g, h->L.total, h->dpart, h->ticket, h->scal + 2);
    KTG_LCUDA(h, cudaMemcpyAsync(h->h_scal + 2, h->scal + 2, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    KTG_LCUDA(h, cudaStreamSynchronize(h->stream));
    const double gn = std::sqrt(h->h_scal[2]);
    const float scale = gn > h->clip ? static_cast<float>(h->clip / gn) : 1.0f;
    ++h->step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, static_cast<float>(h->step));
    const float c2 = 1.0f - std::pow(b2, static_cast<float>(h->step));
    ktg::learned::k_adam<<<static_cast<int>((h->L.total + 255) / 256), 256, 0, h->stream>>>(
        h->w, h->g, h->m1, h->m2, h->L.total, h->lr, b1, b2, 1e-8f, c1, c2, scale);
    h->launches += 2;
    int rc = refresh_bf16(h);
    if (rc) return rc;
    KTG_LCUDA(h, cudaStreamSynchronize(h->stream));
    return KTG_OK;
}

}  // namespace

extern "C" {

int64_t ktg_learned_num_params(void) { return layout().total; }

int ktg_learned_create(int device, uint64_t seed, ktg_learned **out) {
    if (!out) return KTG_ERR_ARG;
    *out = nullptr;
    ktg_learned *h = new (std::nothrow) ktg_learned();
    if (!h) return KTG_ERR_NOMEM;
    h->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return KTG_ERR_CUDA;
    }
    static std::atomic<uint64_t> next_uid{1};
    h->uid = next_uid.fetch_add(1);
    const int64_t P = h->L.total;
    if (lalloc(h, &h->w, P) || lalloc(h, &h->g, P) || lalloc(h, &h->m1, P) ||
        lalloc(h, &h->m2, P) || lalloc(h, &h->wh, P) ||
        lalloc(h, &h->wpart, static_cast<int64_t>(kWgradBlocks) * (HID * HID + HID)) ||
        lalloc(h, &h->dpart, 8192) || lalloc(h, &h->ticket, 1) || lalloc(h, &h->scal, 4) ||
        lalloc(h, &h->tc_status, 1) ||
        cudaMallocHost(&h->h_scal, 4 * sizeof(double)) != cudaSuccess) {
        ktg_learned_destroy(h);
        return KTG_ERR_NOMEM;
    }
    // Glorot-normal init (P scaled by 0.05 so S starts near 0: M ~ Jacobi).
    std::vector<float> w(P, 0.0f);
    uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
    auto unif = [&]() {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        return (static_cast<double>(st >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    };
    auto normal = [&]() { return std::sqrt(-2.0 * std::log(unif())) * std::cos(6.283185307179586 * unif()); };
    auto fill = [&](int64_t ofs, int r, int cdim, double scale) {
        const double sd = std::sqrt(2.0 / (r + cdim)) * scale;
        for (int64_t i = 0; i < static_cast<int64_t>(r) * cdim; ++i) w[ofs + i] = static_cast<float>(normal() * sd);
    };
    const Layout &L = h->L;
    fill(L.W_in, NFEAT, HID, 1.0);
    for (int l = 0; l < LAYERS; ++l) {
        fill(L.Wa[l], HID, HID, 1.0);
        fill(L.Wb[l], HID, HID, 1.0);
        fill(L.Wc[l], HID, HID, 1.0);
    }
    fill(L.P, HID, PROJ, 0.05);
    fill(L.Wh, HEAD_IN, HEAD_H, 1.0);
    fill(L.wz, HEAD_H, 1, 0.1);
    w[L.bz] = static_cast<float>(kSoftplusInvOne);  // untrained head: z = 1 (constant)
    // Every upload is ordered on the handle's stream ahead of the BF16 copy: a
    // plain cudaMemcpy from pageable memory may return before its DMA lands,
    // and the non-blocking stream would not wait for it.
    if (cudaMemcpyAsync(h->w, w.data(), sizeof(float) * P, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaMemsetAsync(h->m1, 0, sizeof(float) * P, h->stream) != cudaSuccess ||
        cudaMemsetAsync(h->m2, 0, sizeof(float) * P, h->stream) != cudaSuccess ||
        cudaMemsetAsync(h->ticket, 0, sizeof(unsigned), h->stream) != cudaSuccess ||
        cudaMemsetAsync(h->tc_status, 0, sizeof(int), h->stream) != cudaSuccess ||
        cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaFuncSetAttribute(ktg::learned::k_dense_umma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             ktg::learned::kUmmaSmem) != cudaSuccess ||
        refresh_bf16(h) != KTG_OK ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
        ktg_learned_destroy(h);
        return KTG_ERR_CUDA;
    }
    *out = h;
    return KTG_OK;
}

void ktg_learned_destroy(ktg_learned *h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    void *ptrs[] = {h->w, h->g, h->m1, h->m2, h->wh, h->x, h->act_c, h->act_n, h->p, h->dp,
                    h->dh, h->dh2, h->dg, h->dm, h->de, h->t, h->ds, h->dphi, h->tr, h->u,
                    h->gq, h->wpart, h->dpart, h->ticket, h->scal, h->tc_status, h->cu, h->chh, h->co,
                    h->cdz, h->cdhh, h->cdo, h->czd, h->caz, h->ce, h->ca, h->cscal};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (h->h_scal) cudaFreeHost(h->h_scal);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

const char *ktg_learned_last_error(const ktg_learned *h) { return h ? h->err.c_str() : "null handle"; }

int ktg_learned_set_option(ktg_learned *h, const char *key, double value) {
    if (!h || !key) return KTG_ERR_ARG;
    const std::string k(key);
    if (k == "tensor_cores" && (value == 0 || value == 1 || value == 2))
        h->tensor_cores = static_cast<int>(value);
    else if (k == "tc_ctas" && value >= 0 && value <= 1 << 20) h->tc_ctas = static_cast<int>(value);
    else if (k == "lr") h->lr = static_cast<float>(value);
    else if (k == "probes" && value >= 1 && value <= 64) h->probes = static_cast<int>(value);
    else if (k == "clip" && value > 0) h->clip = static_cast<float>(value);
    else return lerr(h, KTG_ERR_ARG, "unknown option or value: " + k);
    return KTG_OK;
}

int ktg_learned_get_params(ktg_learned *h, float *out) {
    if (!h || !out) return KTG_ERR_ARG;
    KTG_LCUDA(h, cudaStreamSynchronize(h->stream));
    KTG_LCUDA(h, cudaMemcpy(out, h->w, sizeof(float) * h->L.total, cudaMemcpyDeviceToHost));
    return KTG_OK;
}

int ktg_learned_set_params(ktg_learned *h, const float *in) {
    if (!h || !in) return KTG_ERR_ARG;
    KTG_LCUDA(h, cudaStreamSynchronize(h->stream));
    KTG_LCUDA(h, cudaMemcpyAsync(h->w, in, sizeof(float) * h->L.total, cudaMemcpyHostToDevice,
                                 h->stream));  // stream-ordered ahead of the BF16 copy
    int rc = refresh_bf16(h);
    if (rc) return rc;
    KTG_LCUDA(h, cudaStreamSynchronize(h->stream));
    return KTG_OK;
}

int ktg_learned_loss_grad(ktg_learned *h, ktg_ctx *c, int axis, uint64_t seed, double *loss,
                          float *grad) {
    if (!h || !c || (axis != 0 && axis != 1)) return KTG_ERR_ARG;
    KTG_LCUDA(h, cudaSetDevice(h->device));
    KTG_LCUDA(h, cudaStreamSynchronize(c->stream));
    KTG_LCUDA(h, cudaMemsetAsync(h->g, 0, sizeof(float) * h->L.total, h->stream));
    int rc = loss_grad(h, c, axis, seed, loss);
    if (rc) return rc;
    if (grad) KTG_LCUDA(h, cudaMemcpy(grad, h->g, sizeof(float) * h->L.total, cudaMemcpyDeviceToHost));
    return KTG_OK;
}

int ktg_learned_train_step(ktg_learned *h, ktg_ctx *c, int axis, uint64_t seed, double *loss) {
    double l = 0.0;
    int rc = ktg_learned_loss_grad(h, c, axis, seed, &l, nullptr);
    if (rc) return rc;
    if ((rc = adam_step(h))) return rc;  // global-norm clipped Adam
    if (loss) *loss = l;
    return KTG_OK;
}

int ktg_learned_coarse_loss_grad(ktg_learned *h, ktg_ctx *c, int axis, const double *e,
                                 int32_t num_vec, double *loss, float *grad) {
    if (!h || !c || (axis != 0 && axis != 1) || !e || num_vec < 1 || num_vec > kMaxVec)
        return KTG_ERR_ARG;
    KTG_LCUDA(h, cudaSetDevice(h->device));
    KTG_LCUDA(h, cudaStreamSynchronize(c->stream));
    KTG_LCUDA(h, cudaMemsetAsync(h->g, 0, sizeof(float) * h->L.total, h->stream));
    int rc = coarse_loss_grad(h, c, axis, e, num_vec, loss);
    if (rc) return rc;
    if (grad) KTG_LCUDA(h, cudaMemcpy(grad, h->g, sizeof(float) * h->L.total, cudaMemcpyDeviceToHost));
    return KTG_OK;
}

int ktg_learned_coarse_train_step(ktg_learned *h, ktg_ctx *c, int axis, const double *e,
                                  int32_t num_vec, double *loss) {
    double l = 0.0;
    int rc = ktg_learned_coarse_loss_grad(h, c, axis, e, num_vec, &l, nullptr);
    if (rc) return rc;
    if ((rc = adam_step(h))) return rc;
    if (loss) *loss = l;
    return KTG_OK;
}

int ktg_learned_prepare_coarse(ktg_learned *h, ktg_ctx *c) {
    if (!h || !c) return KTG_ERR_ARG;
    if (!c->have_system || !c->axis_valid[0] || !c->axis_valid[1] || c->sys_n != c->n)
        return lerr(h, KTG_ERR_STATE, "context needs the B2B systems of its netlist");
    KTG_LCUDA(h, cudaSetDevice(h->device));
    const int64_t n = c->n;
    if (!c->coarse_head_w) {  // once per context
        KTG_LCUDA(h, cudaMalloc(&c->coarse_head_w, sizeof(float) * ktg::kCoarseHeadParams));
        KTG_LCUDA(h, cudaMalloc(&c->coarse_logd, 2 * sizeof(double)));
    }
    if (c->coarse_emb_cap < n) {  // the context keeps its netlist's embedding
        if (c->coarse_emb) cudaFree(c->coarse_emb);
        c->coarse_emb = nullptr;
        c->coarse_emb_cap = 0;
        c->coarse_emb_owner = 0;
        KTG_LCUDA(h, cudaMalloc(&c->coarse_emb, sizeof(float) * std::max<int64_t>(n, 1) * PROJ));
        c->coarse_emb_cap = n;
    }
    // Everything below is enqueued on the context's stream.
    cudaStream_t own = h->stream;
    h->stream = c->stream;
    int rc = KTG_OK;
    if (c->coarse_emb_owner != h->uid || c->coarse_emb_gen != c->netlist_gen ||
        c->coarse_emb_version != h->version) {
        rc = topo_trunk(h, c);  // once per netlist and parameter set
        if (!rc && n > 0 && cudaMemcpyAsync(c->coarse_emb, h->p, sizeof(float) * n * PROJ,
                                            cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess)
            rc = lerr(h, KTG_ERR_CUDA, "embedding copy failed");
        if (!rc) {
            c->coarse_emb_owner = h->uid;
            c->coarse_emb_gen = c->netlist_gen;
            c->coarse_emb_version = h->version;
        }
    }
    // the per-axis mean log diagonal and a copy of the head's parameters; the
    // head itself is evaluated per row by the aggregation build
    for (int axis = 0; axis < 2 && !rc; ++axis) {
        const int tb = 256;
        ktg::learned::k_logd_sum<<<std::min<int>(1024, (static_cast<int>(n) + tb - 1) / tb + 1), tb,
                                   0, h->stream>>>(c->sys[axis].diag, static_cast<int32_t>(n),
                                                   h->dpart, h->ticket, c->coarse_logd + axis);
        ++h->launches;
    }
    if (!rc && cudaMemcpyAsync(c->coarse_head_w, h->w + h->L.Wh,
                               sizeof(float) * ktg::kCoarseHeadParams, cudaMemcpyDeviceToDevice,
                               h->stream) != cudaSuccess)
        rc = lerr(h, KTG_ERR_CUDA, "head parameter copy failed");
    h->stream = own;
    if (rc) return rc;
    KTG_LCUDA(h, cudaGetLastError());
    c->coarse_z_ready = true;
    ++c->coarse_z_gen;
    return KTG_OK;
}

int ktg_learned_prepare(ktg_learned *h, ktg_ctx *c) {
    if (!h || !c) return KTG_ERR_ARG;
    KTG_LCUDA(h, cudaSetDevice(h->device));
    KTG_LCUDA(h, cudaStreamSynchronize(c->stream));
    for (int axis = 0; axis < 2; ++axis) {
        SysView S;
        int rc = sys_view(h, c, axis, &S);
        if (rc) return rc;
        if ((rc = forward(h, c, S, c->sys[axis].s32, false))) return rc;
    }
    KTG_LCUDA(h, cudaStreamSynchronize(h->stream));
    c->precond_ready = true;
    return KTG_OK;
}

int64_t ktg_learned_launch_count(const ktg_learned *h) { return h ? h->launches : 0; }

}  // extern "C"
