// Exclusive prefix sums over device arrays: out[0..n] with out[n] = total.
//
// One launch per scan (single pass with decoupled look-back): each block
// takes a ticket from a counter and scans chunk `ticket` of 2048 elements in
// shared memory; it publishes the chunk's total, then walks back over the
// chunks before it, adding published totals until it meets a chunk that has
// published its inclusive prefix, and publishes its own.  A block only waits
// for chunks with lower tickets, which are already running, so the walk
// always ends; the wait is still bounded (about a second) and sets an error
// flag that check_scan_error() reports instead of hanging.  Prefixes are kept in
// 64 bits whatever the element type, so an int32 scan whose total does not
// fit int32 can be detected by the caller (total64).
#include "fmm_internal.cuh"

namespace sfmm {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kChunk = kThreads * kItems;

// chunk state word: status in the top 2 bits (0 nothing, 1 chunk total,
// 2 inclusive prefix), value (non-negative, < 2^62) below
constexpr unsigned long long kStAgg = 1ull << 62, kStPre = 2ull << 62, kValMask = (1ull << 62) - 1;

__device__ int g_scan_error;

__device__ long long block_exclusive64(long long v, long long* total)
{
    __shared__ long long warp_tot[kThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        long long t = lane < kThreads / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < kThreads / 32) warp_tot[lane] = t;
    }
    __syncthreads();
    const long long before = (w ? warp_tot[w - 1] : 0) + x - v;
    *total = warp_tot[kThreads / 32 - 1];
    __syncthreads();
    return before;
}

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// state[0..nb) chunk words, state[nb] the ticket counter; all zero at launch.
// Elements are non-negative counts (the value field holds a 62-bit prefix).
template<typename T>
__global__ void __launch_bounds__(kThreads) k_scan(const T* __restrict__ in, T* __restrict__ out, int64_t n, int64_t nb,
                                                   unsigned long long* state, long long* total64)
{
    __shared__ long long s_chunk, s_prefix;
    if (threadIdx.x == 0) s_chunk = static_cast<long long>(atomicAdd(state + nb, 1ull));
    __syncthreads();
    const int64_t b = s_chunk;
    const int64_t base = b * kChunk + threadIdx.x * kItems;
    T v[kItems];
    long long s = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        v[i] = base + i < n ? in[base + i] : T(0);
        s += static_cast<long long>(v[i]);
    }
    long long agg;
    const long long ex = block_exclusive64(s, &agg);
    if (threadIdx.x == 0) {
        long long prefix = 0;
        if (b == 0) {
            st_release(state, kStPre | (static_cast<unsigned long long>(agg) & kValMask));
        } else {
            st_release(state + b, kStAgg | (static_cast<unsigned long long>(agg) & kValMask));
            int64_t j = b - 1;
            long long spins = 0;
            while (j >= 0) {
                const unsigned long long w = ld_acquire(state + j);
                const unsigned long long st = w & ~kValMask;
                if (st == 0) {
                    if (++spins > (1ll << 22)) {          // ~1 s at the back-off below
                        atomicExch(&g_scan_error, 1);
                        break;
                    }
                    __nanosleep(200);
                    continue;
                }
                prefix += static_cast<long long>(w & kValMask);
                if (st == kStPre) break;
                --j;
            }
            st_release(state + b, kStPre | (static_cast<unsigned long long>(prefix + agg) & kValMask));
        }
        s_prefix = prefix;
        if (b == nb - 1 && total64) *total64 = prefix + agg;
    }
    __syncthreads();
    long long run = s_prefix + ex;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        if (base + i < n) out[base + i] = static_cast<T>(run);
        run += static_cast<long long>(v[i]);
    }
    if (b == nb - 1 && threadIdx.x == kThreads - 1) out[n] = static_cast<T>(run);
}

template<typename T>
__global__ void k_set(T* p, T v, long long* total64)
{
    *p = v;
    if (total64) *total64 = 0;
}

template<typename T>
void exclusive_scan(const T* in, T* out, int64_t n, cudaStream_t s, int64_t* total64)
{
    if (n <= 0) {
        k_set<T><<<1, 1, 0, s>>>(out, T(0), reinterpret_cast<long long*>(total64));
        SFMM_CHECK_LAUNCH();
        return;
    }
    const int64_t nb = (n + kChunk - 1) / kChunk;
    SFMM_REQUIRE(nb < (int64_t(1) << 31), FMM_ERR_UNSUPPORTED, "scan too long");
    DevBuf<unsigned long long> state;
    state.alloc(nb + 1, s);
    SFMM_CUDA(cudaMemsetAsync(state.ptr, 0, size_t(nb + 1) * sizeof(unsigned long long), s));
    k_scan<T><<<static_cast<unsigned>(nb), kThreads, 0, s>>>(in, out, n, nb, state.ptr,
                                                            reinterpret_cast<long long*>(total64));
    SFMM_CHECK_LAUNCH();
}

}  // namespace

void exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, cudaStream_t s, int64_t* total64)
{
    exclusive_scan<int32_t>(in, out, n, s, total64);
}
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s, int64_t* total64)
{
    exclusive_scan<int64_t>(in, out, n, s, total64);
}

void check_scan_error()
{
    int v = 0;
    SFMM_CUDA(cudaMemcpyFromSymbol(&v, g_scan_error, sizeof(int)));
    if (v) {
        const int zero = 0;
        SFMM_CUDA(cudaMemcpyToSymbol(g_scan_error, &zero, sizeof(int)));
        throw Error(FMM_ERR_TIMEOUT, "a prefix sum gave up waiting for an earlier chunk");
    }
}

}  // namespace sfmm
