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
                                                     int64_t chunk, double* __restrict__ part)
{
    __shared__ double s[kThreads][6];
    const int64_t t = blockIdx.x * int64_t(kThreads) + threadIdx.x;
    const bool on = t < nt;
    const int64_t i = on ? targets[t] : 0;
    const double xi = on ? xyz[3 * i] : 0, yi = on ? xyz[3 * i + 1] : 0, zi = on ? xyz[3 * i + 2] : 0;
    double pa[3] = {0, 0, 0}, fa[3] = {0, 0, 0};
    // sources [jb, je) of this block's chunk (blockIdx.y)
    const int64_t jb = blockIdx.y * chunk;
    const int64_t je = jb + chunk < n ? jb + chunk : n;
    for (int64_t j0 = jb; j0 < je; j0 += kThreads) {
        __syncthreads();
        const int64_t j = j0 + threadIdx.x;
        if (j < je) {
            s[threadIdx.x][0] = xyz[3 * j];
            s[threadIdx.x][1] = xyz[3 * j + 1];
            s[threadIdx.x][2] = xyz[3 * j + 2];
            for (int b = 0; b < qdim; ++b) s[threadIdx.x][3 + b] = Q[j * qdim + b];
        }
        __syncthreads();
        const int cnt = je - j0 < kThreads ? static_cast<int>(je - j0) : kThreads;
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
    double* o = part + (blockIdx.y * nt + t) * 6;
    for (int b = 0; b < 3; ++b) o[b] = pa[b];
    for (int c = 0; c < 3; ++c) o[3 + c] = fa[c];
}

// Sum the chunks' partial sums in chunk order (deterministic).
__global__ void k_direct_sum(const double* __restrict__ part, int64_t nt, int nchunk, int qdim,
                             double* __restrict__ pot, double* __restrict__ field)
{
    const int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (t >= nt) return;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int c = 0; c < nchunk; ++c)
        for (int k = 0; k < 6; ++k) acc[k] += part[(c * nt + t) * 6 + k];
    if (pot)
        for (int b = 0; b < qdim; ++b) pot[t * qdim + b] = acc[b];
    if (field)
        for (int c = 0; c < 3; ++c) field[t * 3 + c] = acc[3 + c];
}

}  // namespace

void direct_sum(Context& c, const double* xyz, int64_t n, const double* Q, int qdim, const int64_t* targets, int64_t nt,
                double* pot, double* field)
{
    if (nt <= 0) return;
    // split the sources into chunks so that small target sets still fill the device
    const int64_t gx = (nt + kThreads - 1) / kThreads;
    int64_t nchunk = std::max<int64_t>(1, (int64_t(c.sm_count) * 8 + gx - 1) / gx);
    nchunk = std::min<int64_t>(nchunk, std::max<int64_t>(1, n / (4 * kThreads)));
    nchunk = std::min<int64_t>(nchunk, 65535);
    const int64_t chunk = (n + nchunk - 1) / nchunk;
    DevBuf<double> part;
    part.alloc(size_t(nchunk) * nt * 6, c.stream);
    k_direct<<<dim3(static_cast<unsigned>(gx), static_cast<unsigned>(nchunk)), kThreads, 0, c.stream>>>(
        xyz, n, Q, qdim, targets, nt, chunk, part.ptr);
    SFMM_CHECK_LAUNCH();
    k_direct_sum<<<static_cast<unsigned>((nt + 255) / 256), 256, 0, c.stream>>>(part.ptr, nt, static_cast<int>(nchunk),
                                                                               qdim, pot, field);
    SFMM_CHECK_LAUNCH();
}

}  // namespace sfmm
