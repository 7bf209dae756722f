// Device memory pools: one per device, owned by this library.
#include "fmm_internal.cuh"

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

}  // namespace sfmm
