// Device memory: one pool per device owned by this library, and a cache of
// large blocks in front of it (fmm_internal.cuh describes both).
#include "fmm_internal.cuh"

#include <map>
#include <mutex>

namespace sfmm {

cudaMemPool_t device_pool(int device)
{
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    SFMM_REQUIRE(device >= 0 && device < 64, FMM_ERR_INVALID_ARGUMENT, "device index out of range");
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[device]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        SFMM_CUDA(cudaMemPoolCreate(&pool, &props));
        uint64_t thr = UINT64_MAX;
        SFMM_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
        pools[device] = pool;
    }
    return pools[device];
}

namespace {

constexpr size_t kCacheMin = size_t(4) << 20;

thread_local AllocMeter* tl_meter_request = nullptr;
thread_local AllocMeter* tl_meter_server = nullptr;
thread_local bool tl_cache_on = true;

void meter_add(size_t bytes)
{
    if (tl_meter_request) tl_meter_request->add(int64_t(bytes));
    if (tl_meter_server) tl_meter_server->add(int64_t(bytes));
}

void meter_sub(size_t bytes) noexcept
{
    if (tl_meter_request) tl_meter_request->sub(int64_t(bytes));
    if (tl_meter_server) tl_meter_server->sub(int64_t(bytes));
}

struct Cached {
    void* p;
    cudaEvent_t released;                  // recorded on the releasing stream
    uint64_t age;
};

struct BlockCache {
    std::mutex mu;
    std::multimap<size_t, Cached> blocks;  // by size
    size_t bytes = 0, cap = 0;
    uint64_t clock = 0;
};

BlockCache& block_cache(int device)
{
    static BlockCache caches[64];
    return caches[device];
}

// Frees one cached block once stream s has passed its release.
void drop(std::multimap<size_t, Cached>::iterator it, BlockCache& c, cudaStream_t s) noexcept
{
    (void)cudaStreamWaitEvent(s, it->second.released, 0);
    (void)cudaFreeAsync(it->second.p, s);
    (void)cudaEventDestroy(it->second.released);
    c.bytes -= it->first;
    c.blocks.erase(it);
}

// Restores the caller's current device on scope exit.
struct DeviceScope {
    int old = -1;
    explicit DeviceScope(int device) noexcept
    {
        if (cudaGetDevice(&old) == cudaSuccess && old != device) (void)cudaSetDevice(device);
        else old = -1;
    }
    ~DeviceScope()
    {
        if (old >= 0) (void)cudaSetDevice(old);
    }
};

}  // namespace

void set_thread_alloc_meters(AllocMeter* request, AllocMeter* server) noexcept
{
    tl_meter_request = request;
    tl_meter_server = server;
}

void set_thread_block_cache(bool on) noexcept { tl_cache_on = on; }

void get_thread_alloc_meters(AllocMeter** request, AllocMeter** server) noexcept
{
    *request = tl_meter_request;
    *server = tl_meter_server;
}

bool thread_block_cache() noexcept { return tl_cache_on; }

void* device_alloc(size_t bytes, int device, cudaStream_t s)
{
    SFMM_REQUIRE(device >= 0 && device < 64, FMM_ERR_INVALID_ARGUMENT, "device index out of range");
    BlockCache& c = block_cache(device);
    meter_add(bytes);
    struct Undo {
        size_t b;
        bool armed = true;
        ~Undo()
        {
            if (armed) meter_sub(b);
        }
    } undo{bytes};
    if (bytes >= kCacheMin) {
        std::lock_guard<std::mutex> lk(c.mu);
        auto it = c.blocks.find(bytes);
        if (it != c.blocks.end()) {
            void* p = it->second.p;
            SFMM_CUDA(cudaStreamWaitEvent(s, it->second.released, 0));
            SFMM_CUDA(cudaEventDestroy(it->second.released));
            c.bytes -= bytes;
            c.blocks.erase(it);
            undo.armed = false;
            return p;
        }
    }
    void* p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, device_pool(device), s);
    if (e == cudaErrorMemoryAllocation) {
        (void)cudaGetLastError();
        {
            std::lock_guard<std::mutex> lk(c.mu);
            while (!c.blocks.empty()) drop(c.blocks.begin(), c, s);
        }
        e = cudaMallocFromPoolAsync(&p, bytes, device_pool(device), s);
        if (e == cudaErrorMemoryAllocation) {
            (void)cudaGetLastError();
            throw Error(FMM_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) + " bytes failed");
        }
    }
    SFMM_CUDA(e);
    undo.armed = false;
    return p;
}

void device_free(void* p, size_t bytes, int device, cudaStream_t s) noexcept
{
    if (!p) return;
    meter_sub(bytes);
    if (tl_cache_on && bytes >= kCacheMin && device >= 0 && device < 64) {
        DeviceScope scope(device);
        BlockCache& c = block_cache(device);
        cudaEvent_t ev = nullptr;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess) {
            if (cudaEventRecord(ev, s) == cudaSuccess) {
                std::lock_guard<std::mutex> lk(c.mu);
                if (c.cap == 0) {
                    size_t fr = 0, tot = 0;
                    c.cap = cudaMemGetInfo(&fr, &tot) == cudaSuccess ? tot / 3 : (size_t(8) << 30);
                }
                c.blocks.emplace(bytes, Cached{p, ev, ++c.clock});
                c.bytes += bytes;
                while (c.bytes > c.cap && !c.blocks.empty()) {
                    auto oldest = c.blocks.begin();
                    for (auto it = c.blocks.begin(); it != c.blocks.end(); ++it)
                        if (it->second.age < oldest->second.age) oldest = it;
                    drop(oldest, c, s);
                }
                return;
            }
            (void)cudaEventDestroy(ev);
        }
        (void)cudaGetLastError();
    }
    (void)cudaFreeAsync(p, s);
}

}  // namespace sfmm
