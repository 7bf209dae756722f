// Device helpers shared by the evaluation kernels.
#pragma once

#include "fmm_eval.cuh"

namespace sfmm {

static __device__ __forceinline__ int level_of(const EvalArgs& a, int64_t g)
{
    int l = 0;
    while (l < a.depth && g >= a.lvl_off[l + 1]) ++l;
    return l;
}

// box.hpp:147-150
static __device__ __forceinline__ void node_center(const BoxDev& b, uint64_t key, int l, double* c)
{
    const uint32_t ix = compact3(key), iy = compact3(key >> 1), iz = compact3(key >> 2);
    const double s = double(1 << l);
    c[0] = b.corner[0] + b.width * ((ix + 0.5) / s);
    c[1] = b.corner[1] + b.width * ((iy + 0.5) / s);
    c[2] = b.corner[2] + b.width * ((iz + 0.5) / s);
}

static __device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

static __device__ __forceinline__ void tri_nm(int t, int& n, int& m)
{
    n = static_cast<int>((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
    if ((n + 1) * (n + 2) / 2 <= t) ++n;
    if (n * (n + 1) / 2 > t) --n;
    m = t - n * (n + 1) / 2;
}


// M2L over all sibling groups (children of nodes in [g0, g1)), m2l.cu.
void launch_m2l(const EvalArgs& a, int64_t g0, int64_t g1, int sms, cudaStream_t st);
// The same with the direct (dense) formulation, m2l_direct.cu.
void launch_m2l_direct(const EvalArgs& a, int64_t g0, int64_t g1, int sms, cudaStream_t st);

// Near field of every leaf into a.out2, p2p.cu.
void launch_p2p(const EvalArgs& a, int sms, cudaStream_t st);

}  // namespace sfmm
