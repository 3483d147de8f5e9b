// The head of the learned coarse vector, shared by the network's own kernels
// (training, ktg_learned.cu) and the aggregation build that evaluates it per
// permuted row (ktg_agg.cu):
//   z_i = softplus(relu(u_i Wh + bh) . wz + bz),   u_i = (p_i, c_i, l_i)
// with p_i the cell's 16-wide trunk embedding, c_i = sum_j |a_ij| / a_ii the
// coupling share and l_i = log a_ii - mean log a (FP64, then rounded). The
// parameters are packed as Wh [18 x 16] | bh [16] | wz [16] | bz, the order
// they have in the network's parameter vector. One evaluation order is used
// everywhere, so training and inference give the same z.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ktg {

constexpr int kCoarseProj = 16;                 // trunk embedding width
constexpr int kCoarseIn = kCoarseProj + 2;      // head inputs
constexpr int kCoarseHid = 16;                  // head hidden width
constexpr int kCoarseHeadParams = kCoarseIn * kCoarseHid + 2 * kCoarseHid + 1;

// Pre-softplus output o of the head for inputs u; ws the packed parameters.
template <class Load>
__device__ __forceinline__ float coarse_head_o(const float (&u)[kCoarseIn], Load ws) {
    float o = ws(kCoarseIn * kCoarseHid + 2 * kCoarseHid);
#pragma unroll
    for (int j = 0; j < kCoarseHid; ++j) {
        float t = ws(kCoarseIn * kCoarseHid + j);
#pragma unroll
        for (int k = 0; k < kCoarseIn; ++k) t += u[k] * ws(k * kCoarseHid + j);
        t = t > 0.0f ? t : 0.0f;
        o += t * ws(kCoarseIn * kCoarseHid + kCoarseHid + j);
    }
    return o;
}

__device__ __forceinline__ float coarse_softplus(float o) {
    return o > 20.0f ? o : log1pf(expf(o));
}

// z of one row from its embedding, the FP64 sum of |a_ij| over its
// off-diagonal entries, its diagonal and the axis's mean log diagonal.
template <class Load>
__device__ __forceinline__ float coarse_head_z(const float *p, double rowabs, double d,
                                               double logd_mean, Load ws) {
    float u[kCoarseIn];
#pragma unroll
    for (int k = 0; k < kCoarseProj; ++k) u[k] = __ldg(p + k);
    u[kCoarseProj] = static_cast<float>(rowabs / d);
    u[kCoarseProj + 1] = static_cast<float>(log(d) - logd_mean);
    return coarse_softplus(coarse_head_o(u, ws));
}

}  // namespace ktg
