// Direct FP64 sums at selected targets -- the reference's accuracy check
// (main.cpp:70-111) on the device: thread per target, source tiles staged
// in shared memory.  Used to state the FMM error against the exact sum.
#include "fmm_internal.cuh"

namespace sfmm {

std::atomic<long long> g_launches{0};

namespace {

constexpr int kThreads = 128;

__global__ void __launch_bounds__(kThreads) k_direct(const double* __restrict__ xyz, int64_t n,
                                                     const double* __restrict__ Q, int qdim,
                                                     const int64_t* __restrict__ targets, int64_t nt,
                                                     double* __restrict__ pot, double* __restrict__ field)
{
    __shared__ double s[kThreads][6];
    const int64_t t = blockIdx.x * int64_t(kThreads) + threadIdx.x;
    const bool on = t < nt;
    const int64_t i = on ? targets[t] : 0;
    const double xi = on ? xyz[3 * i] : 0, yi = on ? xyz[3 * i + 1] : 0, zi = on ? xyz[3 * i + 2] : 0;
    double pa[3] = {0, 0, 0}, fa[3] = {0, 0, 0};
    for (int64_t j0 = 0; j0 < n; j0 += kThreads) {
        __syncthreads();
        const int64_t j = j0 + threadIdx.x;
        if (j < n) {
            s[threadIdx.x][0] = xyz[3 * j];
            s[threadIdx.x][1] = xyz[3 * j + 1];
            s[threadIdx.x][2] = xyz[3 * j + 2];
            for (int b = 0; b < qdim; ++b) s[threadIdx.x][3 + b] = Q[j * qdim + b];
        }
        __syncthreads();
        const int cnt = n - j0 < kThreads ? static_cast<int>(n - j0) : kThreads;
        if (!on) continue;
        for (int k = 0; k < cnt; ++k) {
            if (j0 + k == i) continue;
            const double dx = xi - s[k][0], dy = yi - s[k][1], dz = zi - s[k][2];
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            const double r3 = r * r * r;
            for (int b = 0; b < qdim; ++b) pa[b] += s[k][3 + b] / r;
            if (qdim == 1) {
                fa[0] += s[k][3] * dx / r3;
                fa[1] += s[k][3] * dy / r3;
                fa[2] += s[k][3] * dz / r3;
            } else if (qdim == 3) {
                fa[0] += (s[k][4] * dz - s[k][5] * dy) / r3;
                fa[1] += (s[k][5] * dx - s[k][3] * dz) / r3;
                fa[2] += (s[k][3] * dy - s[k][4] * dx) / r3;
            }
        }
    }
    if (!on) return;
    if (pot)
        for (int b = 0; b < qdim; ++b) pot[t * qdim + b] = pa[b];
    if (field)
        for (int c = 0; c < 3; ++c) field[t * 3 + c] = fa[c];
}

}  // namespace

void direct_sum(Context& c, const double* xyz, int64_t n, const double* Q, int qdim, const int64_t* targets, int64_t nt,
                double* pot, double* field)
{
    if (nt <= 0) return;
    k_direct<<<static_cast<unsigned>((nt + kThreads - 1) / kThreads), kThreads, 0, c.stream>>>(xyz, n, Q, qdim, targets,
                                                                                                nt, pot, field);
    SFMM_CHECK_LAUNCH();
}

}  // namespace sfmm
