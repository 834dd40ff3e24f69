// memory.cuh -- device and pinned-host memory for the solvers.
//
// Device memory comes from one library-owned stream-ordered pool per device
// (cudaMemPoolCreate) whose release threshold keeps freed blocks cached for
// the next solve, so a one-shot solve pays no cudaMalloc.  Control-block
// mirrors come from one pinned-host slab carved into 256-byte slots.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "common.cuh"

namespace rb200 {

cudaError_t pool_alloc(void** ptr, size_t bytes, cudaStream_t stream);
void* pinned_get();          // a 256-byte pinned slot, or nullptr
void pinned_put(void* slot);

// A non-blocking stream of the current device (*device receives it) from a
// library-owned pool, created on first need; stream_put returns it, idle (the
// caller has synchronised it), for the next solver.  A one-shot solve then
// pays no stream creation or destruction.
cudaError_t stream_get(cudaStream_t* out, int* device);
void stream_put(cudaStream_t s, int device);

// Host-to-device copies of caller (pageable) memory through a library-owned
// pinned staging ring: host threads fill one slot while the copy engine drains
// the other, so the copy runs at the pinned rate instead of the driver's
// pageable one.  Each call returns once its last chunk is queued on `stream`;
// the caller's memory is no longer read after that.  Calls from several host
// threads take turns.
cudaError_t staged_upload(void* dst, const void* src, size_t bytes, cudaStream_t stream);

// Device-to-host copy of `count` values into caller (pageable) memory as
// doubles, through the same pinned ring: the copy engine fills one slot
// while the host threads widen the other into dst, so the caller's pages are
// first touched by several threads at once and no host staging vector is
// allocated.  Returns once dst is complete (the stream is synchronised up to
// the last chunk's copy).
cudaError_t staged_download_as_double(double* dst, const float* src, size_t count, cudaStream_t stream);
cudaError_t staged_download_as_double(double* dst, const double* src, size_t count, cudaStream_t stream);
// The same for `bytes` copied as they are.  Both return
// cudaErrorMemoryAllocation, having copied nothing, when no pinned ring can
// be had.
cudaError_t staged_download(void* dst, const void* src, size_t bytes, cudaStream_t stream);

template <class T>
struct PoolBuf {
    T* ptr = nullptr;
    size_t count = 0;
    cudaStream_t stream = nullptr;
    PoolBuf() = default;
    PoolBuf(const PoolBuf&) = delete;
    PoolBuf& operator=(const PoolBuf&) = delete;
    ~PoolBuf() { release(); }
    void release() {
        if (ptr) cudaFreeAsync(ptr, stream);
        ptr = nullptr;
        count = 0;
    }
    cudaError_t alloc(size_t n, cudaStream_t s) {
        release();
        stream = s;
        count = n;
        return pool_alloc(reinterpret_cast<void**>(&ptr), sizeof(T) * n, s);
    }
    cudaError_t upload(const T* host, size_t n, cudaStream_t s) {
        RB_CUDA_TRY(alloc(n, s));
        if (n) RB_CUDA_TRY(cudaMemcpyAsync(ptr, host, sizeof(T) * n, cudaMemcpyHostToDevice, s));
        return cudaSuccess;
    }
};

}  // namespace rb200
