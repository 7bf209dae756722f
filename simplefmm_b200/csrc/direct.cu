// Direct FP64 sums at selected targets -- the reference's accuracy check
// (main.cpp:70-111) on the device: thread per target, source tiles staged
// in shared memory.  Used to state the FMM error against the exact sum.
#include "fmm_internal.cuh"

#include <mutex>

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
    const int64_t ti = t < nt ? targets[t] : -1;
    // a target index outside [0, n) reads nothing; k_direct_sum reports it
    const bool on = ti >= 0 && ti < n;
    const int64_t i = on ? ti : 0;
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

// Sum the chunks' partial sums in chunk order (deterministic).  A target
// index outside [0, n) gets NaN outputs and sets *bad (when given).
__global__ void k_direct_sum(const double* __restrict__ part, int64_t nt, int nchunk, int qdim,
                             const int64_t* __restrict__ targets, int64_t n, double* __restrict__ pot,
                             double* __restrict__ field, int* __restrict__ bad)
{
    const int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (t >= nt) return;
    const int64_t ti = targets[t];
    if (ti < 0 || ti >= n) {
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        if (pot)
            for (int b = 0; b < qdim; ++b) pot[t * qdim + b] = nan;
        if (field)
            for (int c = 0; c < 3; ++c) field[t * 3 + c] = nan;
        if (bad) atomicOr(bad, 1);
        return;
    }
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
                double* pot, double* field, int* bad)
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
    k_direct_sum<<<static_cast<unsigned>((nt + 255) / 256), 256, 0, c.stream>>>(
        part.ptr, nt, static_cast<int>(nchunk), qdim, targets, n, pot, field, bad);
    SFMM_CHECK_LAUNCH();
}

}  // namespace sfmm

// ------------------------------------------------------------------ direct sum without allocation
// fmm_direct_noalloc: the same two kernels with their partial sums in a
// fixed, file-scope device array instead of memory allocated per call.  It is
// for callers that cannot allocate device memory while they run: callers that
// hold a fixed device-memory budget for their own lifetime (a solver service
// that admits work against a budget), and callers that cannot wait on an
// allocation (growing a memory pool can stall a call for a long time).
namespace sfmm {
namespace {

// Partial sums: 6 doubles per (source chunk, target).  8 MiB on every device
// that loads this library, held until the process exits.
constexpr int64_t kNoAllocScratchDoubles = int64_t(1) << 20;
constexpr int64_t kNoAllocMaxTargets = kNoAllocScratchDoubles / 6;    // 174,762
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

struct NoAllocDevice {
    double* scratch = nullptr;     // device address of g_noalloc_scratch
    int sms = 0;
};

// Set-up, once per device, with that device current: the device address of
// the scratch array (its host-side name is only a stand-in) and the SM count.
NoAllocDevice noalloc_device(int dev)
{
    static std::mutex mu;
    static NoAllocDevice table[64];
    std::lock_guard<std::mutex> lk(mu);
    NoAllocDevice& d = table[dev];
    if (!d.scratch) {
        double* ptr = nullptr;
        SFMM_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_noalloc_scratch));
        int sms = 0;
        SFMM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        d.sms = sms;
        d.scratch = ptr;
    }
    return d;
}

}  // namespace
}  // namespace sfmm

extern "C" int fmm_direct_noalloc(const double* xyz, int64_t n, const double* Q, int qdim, const int64_t* targets,
                                  int64_t nt, double* pot, double* field, void* stream)
{
    using namespace sfmm;
    try {
        if (!xyz || !Q || !targets) return record_failure(FMM_ERR_INVALID_ARGUMENT, "NULL argument");
        if (qdim < 1 || qdim > 3) return record_failure(FMM_ERR_UNSUPPORTED, "qdim must be 1, 2 or 3");
        if (field && qdim == 2) return record_failure(FMM_ERR_UNSUPPORTED, "the field needs qdim 1 or 3");
        if (n <= 0 || nt < 0) return record_failure(FMM_ERR_INVALID_ARGUMENT, "bad sizes");
        if (nt > kNoAllocMaxTargets)
            return record_failure(FMM_ERR_OVER_BUDGET,
                                  "fmm_direct_noalloc takes at most 174762 targets per call (8 MiB of fixed scratch)");
        if (nt == 0) return FMM_OK;
        int dev = 0;
        SFMM_CUDA(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 64) return record_failure(FMM_ERR_UNSUPPORTED, "device index above 63");
        const NoAllocDevice d = noalloc_device(dev);
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        // chunking as direct_sum, capped by the scratch size
        const int64_t gx = (nt + kThreads - 1) / kThreads;
        int64_t nchunk = std::max<int64_t>(1, (int64_t(d.sms) * 8 + gx - 1) / gx);
        nchunk = std::min<int64_t>(nchunk, std::max<int64_t>(1, n / (4 * kThreads)));
        nchunk = std::min<int64_t>(nchunk, kNoAllocScratchDoubles / (6 * nt));
        nchunk = std::min<int64_t>(nchunk, 65535);
        const int64_t chunk = (n + nchunk - 1) / nchunk;
        // every (chunk, target) slot of the scratch is written before it is
        // read, so nothing left by an earlier call needs clearing
        k_direct<<<dim3(static_cast<unsigned>(gx), static_cast<unsigned>(nchunk)), kThreads, 0, st>>>(
            xyz, n, Q, qdim, targets, nt, chunk, d.scratch);
        SFMM_CHECK_LAUNCH();
        // a target index outside [0, n) is not read: its outputs become NaN
        k_direct_sum<<<static_cast<unsigned>((nt + 255) / 256), 256, 0, st>>>(
            d.scratch, nt, static_cast<int>(nchunk), qdim, targets, n, pot, field, nullptr);
        SFMM_CHECK_LAUNCH();
        return FMM_OK;
    } catch (const sfmm::Error& e) {
        return record_failure(e.status, e.what());
    } catch (const std::exception& e) {
        return record_failure(FMM_ERR_CUDA, e.what());
    }
}
