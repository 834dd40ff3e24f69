// memory.cu -- the pools declared in memory.cuh.
#include "memory.cuh"

#include <cstdint>
#include <mutex>
#include <vector>

namespace rb200 {

static cudaError_t pool_for_current_device(cudaMemPool_t* out) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    RB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool;
        RB_CUDA_TRY(cudaMemPoolCreate(&pool, &props));
        uint64_t keep = ~uint64_t(0);
        RB_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        pools[dev] = pool;
    }
    *out = pools[dev];
    return cudaSuccess;
}

cudaError_t pool_alloc(void** ptr, size_t bytes, cudaStream_t stream) {
    cudaMemPool_t pool;
    RB_CUDA_TRY(pool_for_current_device(&pool));
    return cudaMallocFromPoolAsync(ptr, bytes ? bytes : 16, pool, stream);
}

namespace {
constexpr int kSlot = 256, kSlots = 4096;
std::mutex slab_mu;
char* slab_base = nullptr;
std::vector<int> slab_free;
}  // namespace

void* pinned_get() {
    std::lock_guard<std::mutex> lock(slab_mu);
    if (!slab_base) {
        if (cudaHostAlloc(reinterpret_cast<void**>(&slab_base), size_t(kSlot) * kSlots,
                          cudaHostAllocPortable) != cudaSuccess) {
            slab_base = nullptr;
            return nullptr;
        }
        for (int k = kSlots - 1; k >= 0; --k) slab_free.push_back(k);
    }
    if (slab_free.empty()) return nullptr;
    const int k = slab_free.back();
    slab_free.pop_back();
    return slab_base + size_t(k) * kSlot;
}

void pinned_put(void* slot) {
    if (!slot) return;
    std::lock_guard<std::mutex> lock(slab_mu);
    slab_free.push_back(int((static_cast<char*>(slot) - slab_base) / kSlot));
}

}  // namespace rb200
