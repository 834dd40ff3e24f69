// memory.cu -- the pools declared in memory.cuh.
#include "memory.cuh"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
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

namespace {
std::mutex streams_mu;
std::vector<cudaStream_t> idle_streams[64];
}  // namespace

cudaError_t stream_get(cudaStream_t* out, int* device) {
    int dev = 0;
    RB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    *device = dev;
    {
        std::lock_guard<std::mutex> lock(streams_mu);
        if (!idle_streams[dev].empty()) {
            *out = idle_streams[dev].back();
            idle_streams[dev].pop_back();
            return cudaSuccess;
        }
    }
    return cudaStreamCreateWithFlags(out, cudaStreamNonBlocking);
}

void stream_put(cudaStream_t s, int device) {
    if (!s || device < 0 || device >= 64) return;
    std::lock_guard<std::mutex> lock(streams_mu);
    idle_streams[device].push_back(s);
}

}  // namespace rb200

// --- staged host-to-device copies ---------------------------------------------

namespace rb200 {
namespace {

// A fixed set of host threads that run one job at a time: parallel(f) calls
// f(k) once for every k = 0 .. size-1 and returns when all calls have
// returned.  The parts are claimed from a counter by the calling thread and
// by whichever helpers wake while the job is open, so a helper that the
// system does not schedule in time (other processes on the host) holds
// nothing up: its parts go to the others, and once every part is claimed the
// job closes and the caller waits only for the helpers that joined it.
// Started on first use, joined at exit.
class HostThreads {
public:
    explicit HostThreads(int helpers) : helpers_(helpers) {
        for (int k = 1; k <= helpers_; ++k) threads_.emplace_back([this] { loop(); });
    }
    ~HostThreads() {
        {
            std::lock_guard<std::mutex> lock(mu_);
            stop_ = true;
        }
        wake_.notify_all();
        for (auto& t : threads_) t.join();
    }
    int size() const { return helpers_ + 1; }
    void parallel(const std::function<void(int)>& f) {
        {
            std::lock_guard<std::mutex> lock(mu_);
            job_ = &f;
            parts_ = size();
            next_.store(0, std::memory_order_relaxed);
            open_ = true;
            ++generation_;
        }
        wake_.notify_all();
        run_parts(f);
        std::unique_lock<std::mutex> lock(mu_);
        open_ = false;   // every part is claimed: no helper joins from here on
        done_.wait(lock, [this] { return active_ == 0; });
        job_ = nullptr;
    }

private:
    void run_parts(const std::function<void(int)>& f) {
        for (int k; (k = next_.fetch_add(1, std::memory_order_relaxed)) < parts_;) f(k);
    }
    void loop() {
        long long seen = 0;
        for (;;) {
            const std::function<void(int)>* f;
            {
                std::unique_lock<std::mutex> lock(mu_);
                wake_.wait(lock, [&] { return stop_ || (open_ && generation_ != seen); });
                if (stop_) return;
                seen = generation_;
                f = job_;
                ++active_;
            }
            run_parts(*f);
            std::lock_guard<std::mutex> lock(mu_);
            if (--active_ == 0) done_.notify_all();
        }
    }
    int helpers_;
    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable wake_, done_;
    const std::function<void(int)>* job_ = nullptr;
    int parts_ = 0;
    std::atomic<int> next_{0};
    long long generation_ = 0;
    int active_ = 0;
    bool open_ = false;
    bool stop_ = false;
};

HostThreads& host_threads() {
    static HostThreads pool(std::max(0, std::min(7, int(std::thread::hardware_concurrency()) - 1)));
    return pool;
}

constexpr size_t kStageBytes = size_t(4) << 20;   // per slot; two slots
std::mutex stage_mu;
char* stage_ring = nullptr;
cudaEvent_t stage_done[64][2] = {};                 // per device and slot
int stage_dev[2] = {-1, -1};                        // the device whose copy last read each slot

// Copies `bytes` of output to dst in chunks: fill(chunk_dst_host, first_byte,
// chunk_bytes) writes a chunk into a pinned slot, split over the host threads.
template <class Fill>
cudaError_t staged(char* dst, size_t bytes, size_t unit, cudaStream_t stream, Fill fill) {
    if (!bytes) return cudaSuccess;
    std::lock_guard<std::mutex> lock(stage_mu);
    int dev = 0;
    RB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!stage_ring && cudaHostAlloc(reinterpret_cast<void**>(&stage_ring), 2 * kStageBytes,
                                     cudaHostAllocPortable) != cudaSuccess) {
        stage_ring = nullptr;
        (void)cudaGetLastError();
        return cudaErrorMemoryAllocation;   // the caller copies directly instead
    }
    for (auto& ev : stage_done[dev])
        if (!ev) RB_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    HostThreads& pool = host_threads();
    const size_t chunk = kStageBytes / unit * unit;
    int slot = 0;
    for (size_t off = 0; off < bytes; off += chunk, slot ^= 1) {
        const size_t len = std::min(chunk, bytes - off);
        char* buf = stage_ring + size_t(slot) * kStageBytes;
        if (stage_dev[slot] >= 0)   // the slot's last copy, from whichever device, is done
            RB_CUDA_TRY(cudaEventSynchronize(stage_done[stage_dev[slot]][slot]));
        const size_t units = len / unit, parts = size_t(pool.size());
        pool.parallel([&](int k) {
            const size_t a = units * size_t(k) / parts, b = units * size_t(k + 1) / parts;
            if (b > a) fill(buf + a * unit, off + a * unit, (b - a) * unit);
        });
        RB_CUDA_TRY(cudaMemcpyAsync(dst + off, buf, len, cudaMemcpyHostToDevice, stream));
        RB_CUDA_TRY(cudaEventRecord(stage_done[dev][slot], stream));
        stage_dev[slot] = dev;
    }
    return cudaSuccess;
}

// Copies `bytes` of device memory at src back in chunks through the ring:
// chunk c + 1 is copied while drain(first_unit, units, slot) hands chunk c on,
// split over the host threads (on the calling thread alone for small chunks).
template <class Drain>
cudaError_t staged_back(const char* src, size_t bytes, size_t unit, cudaStream_t stream, Drain drain) {
    if (!bytes) return cudaSuccess;
    std::lock_guard<std::mutex> lock(stage_mu);
    int dev = 0;
    RB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!stage_ring && cudaHostAlloc(reinterpret_cast<void**>(&stage_ring), 2 * kStageBytes,
                                     cudaHostAllocPortable) != cudaSuccess) {
        stage_ring = nullptr;
        (void)cudaGetLastError();
        return cudaErrorMemoryAllocation;
    }
    for (auto& ev : stage_done[dev])
        if (!ev) RB_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    const size_t chunk = kStageBytes / unit * unit;
    const size_t chunks = (bytes + chunk - 1) / chunk;
    auto issue = [&](size_t c) -> cudaError_t {
        const int slot = int(c & 1);
        if (stage_dev[slot] >= 0)   // the slot's last copy, from whichever device, is done
            RB_CUDA_TRY(cudaEventSynchronize(stage_done[stage_dev[slot]][slot]));
        const size_t off = c * chunk, len = std::min(chunk, bytes - off);
        RB_CUDA_TRY(cudaMemcpyAsync(stage_ring + size_t(slot) * kStageBytes, src + off, len,
                                    cudaMemcpyDeviceToHost, stream));
        RB_CUDA_TRY(cudaEventRecord(stage_done[dev][slot], stream));
        stage_dev[slot] = dev;
        return cudaSuccess;
    };
    RB_CUDA_TRY(issue(0));
    HostThreads& pool = host_threads();
    constexpr size_t kAloneUnits = size_t(1) << 15;   // below this a chunk is drained on one thread
    for (size_t c = 0; c < chunks; ++c) {
        if (c + 1 < chunks) RB_CUDA_TRY(issue(c + 1));
        const int slot = int(c & 1);
        RB_CUDA_TRY(cudaEventSynchronize(stage_done[dev][slot]));
        const char* buf = stage_ring + size_t(slot) * kStageBytes;
        const size_t first = c * chunk / unit, units = std::min(chunk, bytes - c * chunk) / unit;
        if (units < kAloneUnits) {
            drain(first, units, buf);
            continue;
        }
        const size_t parts = size_t(pool.size());
        pool.parallel([&](int k) {
            const size_t a = units * size_t(k) / parts, b = units * size_t(k + 1) / parts;
            if (b > a) drain(first + a, b - a, buf + a * unit);
        });
    }
    return cudaSuccess;
}

template <class T>
cudaError_t download_as_double(double* dst, const T* src, size_t count, cudaStream_t stream) {
    return staged_back(reinterpret_cast<const char*>(src), sizeof(T) * count, sizeof(T), stream,
                       [dst](size_t first, size_t units, const char* from) {
                           const T* v = reinterpret_cast<const T*>(from);
                           double* out = dst + first;
                           for (size_t k = 0; k < units; ++k) out[k] = double(v[k]);
                       });
}

}  // namespace

cudaError_t staged_download_as_double(double* dst, const float* src, size_t count, cudaStream_t stream) {
    return download_as_double(dst, src, count, stream);
}

cudaError_t staged_download_as_double(double* dst, const double* src, size_t count, cudaStream_t stream) {
    return download_as_double(dst, src, count, stream);
}

cudaError_t staged_download(void* dst, const void* src, size_t bytes, cudaStream_t stream) {
    char* out = static_cast<char*>(dst);
    return staged_back(static_cast<const char*>(src), bytes, 1, stream,
                       [out](size_t first, size_t len, const char* from) { std::memcpy(out + first, from, len); });
}

cudaError_t staged_upload(void* dst, const void* src, size_t bytes, cudaStream_t stream) {
    const char* s = static_cast<const char*>(src);
    const cudaError_t st = staged(static_cast<char*>(dst), bytes, 1, stream,
                                  [s](char* out, size_t first, size_t len) { std::memcpy(out, s + first, len); });
    // no pinned ring to be had: the driver's own (pageable) copy
    if (st == cudaErrorMemoryAllocation) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);
    return st;
}

}  // namespace rb200
