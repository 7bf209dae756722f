// Exclusive prefix sums over device arrays: out[0..n] with out[n] = total.
// Three phases: per-chunk totals, one-block scan of the totals (with a carry
// loop, any number of chunks), per-chunk scan seeded with its offset.
#include "fmm_internal.cuh"

namespace sfmm {
namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kChunk = kThreads * kItems;

template<typename T>
__device__ T block_exclusive(T v, T* total)
{
    __shared__ T warp_tot[kThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        T t = lane < kThreads / 32 ? warp_tot[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < kThreads / 32) warp_tot[lane] = t;
    }
    __syncthreads();
    const T before = (w ? warp_tot[w - 1] : T(0)) + x - v;
    *total = warp_tot[kThreads / 32 - 1];
    __syncthreads();
    return before;
}

template<typename T>
__global__ void k_chunk_sums(const T* in, int64_t n, T* sums)
{
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kChunk + threadIdx.x * kItems;
    T s = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i)
        if (base + i < n) s += in[base + i];
    T tot;
    block_exclusive(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

template<typename T>
__global__ void k_scan_sums(T* sums, int64_t nb)
{
    T carry = 0;
    for (int64_t b0 = 0; b0 < nb; b0 += kThreads) {
        const int64_t i = b0 + threadIdx.x;
        const T v = i < nb ? sums[i] : T(0);
        T tot;
        const T ex = block_exclusive(v, &tot);
        if (i < nb) sums[i] = carry + ex;
        carry += tot;
    }
}

template<typename T>
__global__ void k_chunk_scan(const T* in, T* out, int64_t n, const T* offs, int64_t nb)
{
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kChunk + threadIdx.x * kItems;
    T v[kItems];
    T s = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        v[i] = base + i < n ? in[base + i] : T(0);
        s += v[i];
    }
    T tot;
    T run = block_exclusive(s, &tot) + offs[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
    if (blockIdx.x == nb - 1 && threadIdx.x == kThreads - 1) out[n] = run;
}

template<typename T>
__global__ void k_set(T* p, T v) { *p = v; }

template<typename T>
void exclusive_scan(const T* in, T* out, int64_t n, cudaStream_t s)
{
    if (n <= 0) {
        k_set<T><<<1, 1, 0, s>>>(out, T(0));
        SFMM_CHECK_LAUNCH();
        return;
    }
    const int64_t nb = (n + kChunk - 1) / kChunk;
    DevBuf<T> sums;
    sums.alloc(nb, s);
    k_chunk_sums<T><<<static_cast<unsigned>(nb), kThreads, 0, s>>>(in, n, sums.ptr);
    SFMM_CHECK_LAUNCH();
    k_scan_sums<T><<<1, kThreads, 0, s>>>(sums.ptr, nb);
    SFMM_CHECK_LAUNCH();
    k_chunk_scan<T><<<static_cast<unsigned>(nb), kThreads, 0, s>>>(in, out, n, sums.ptr, nb);
    SFMM_CHECK_LAUNCH();
}

}  // namespace

void exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, cudaStream_t s) { exclusive_scan<int32_t>(in, out, n, s); }
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s) { exclusive_scan<int64_t>(in, out, n, s); }

}  // namespace sfmm
