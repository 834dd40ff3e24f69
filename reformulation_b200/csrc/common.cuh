// common.cuh -- shared device/host helpers for the PRAQ and PRIA solvers.
//
// Everything here is plain sm_100a CUDA C++: warp shuffles, shared memory and
// fixed-order block reductions (deterministic: the order of additions depends
// on the launch shape only, so a solve is bitwise reproducible run to run).
#pragma once

#include <utility>

#include <cuda_runtime.h>

#include "../../include/reform_trace.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <limits>
#include <mutex>
#include <vector>

namespace rb200 {

constexpr int kWarp = 32;

#define RB_CUDA_TRY(call)                                      \
    do {                                                       \
        cudaError_t rb_err_ = (call);                          \
        if (rb_err_ != cudaSuccess) return rb_err_;            \
    } while (0)

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum K doubles over the block; the total lands in out[0..K) (written by
// thread 0).  Fixed order: butterfly within each warp, then warp 0 adds the
// per-warp totals in warp order.  `scratch` holds K * 32 doubles.
template <int K>
__device__ __forceinline__ void block_sums(double (&v)[K], double* scratch, double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int warps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = warp_sum(v[k]);
        if (lane == 0) scratch[k * 32 + warp] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = lane < warps ? scratch[k * 32 + lane] : 0.0;
            s = warp_sum(s);
            if (lane == 0) out[k] = s;
        }
    }
    __syncthreads();
}

// Deterministic sum of `count` rows of K doubles (row-major, stride K) by one
// block: thread t adds rows t, t + blockDim, ... in order, then block_sums.
// A thread's rows are loaded four at a time by predicated loads, so each
// group of four costs one memory round trip.
template <int K>
__device__ __forceinline__ void reduce_rows(const double* rows, int count, double* scratch,
                                            double* out) {
    constexpr int kRows = 4;
    double v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = 0.0;
    for (int r0 = threadIdx.x; r0 < count; r0 += kRows * blockDim.x) {
        double t[kRows][K];
#pragma unroll
        for (int u = 0; u < kRows; ++u) {
            const int r = r0 + u * int(blockDim.x);
            if (r < count) {
#pragma unroll
                for (int k = 0; k < K; ++k) t[u][k] = rows[size_t(r) * K + k];
            }
        }
#pragma unroll
        for (int u = 0; u < kRows; ++u) {
            if (r0 + u * int(blockDim.x) < count) {
#pragma unroll
                for (int k = 0; k < K; ++k) v[k] += t[u][k];
            }
        }
    }
    block_sums<K>(v, scratch, out);
}

// Programmatic dependent launch: a kernel launched with the programmatic
// stream-serialization attribute may start before the kernel ahead of it on
// the stream has finished.  pdl_wait() blocks until that kernel has completed
// and its memory is visible (a no-op for a kernel launched without the
// attribute); pdl_launch_dependents() lets the next kernel start its CTAs as
// soon as every CTA of this one has issued it.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;"); }

// Launch `kernel` on `stream` with the programmatic stream-serialization
// attribute (the kernel must call pdl_wait() before it touches memory the
// previous kernel writes).
template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), int grid, int block, cudaStream_t stream, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(unsigned(block));
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Start bringing the line of `p` into L2 (no register, no wait): for data a
// later pass of the same thread block reads, so that pass finds it on chip.
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// ---- the grid barrier of a persistent (cooperative) launch -----------------
// Every CTA arrives once per barrier; the last to arrive resets the count and
// advances the generation the others wait on.  Waits are bounded: a CTA that
// has waited `limit_ns` of %globaltimer, or that sees `err` set, sets `err`
// and gives up, so a barrier that cannot complete ends the kernel with an
// error the host reads (and clears before the next launch) instead of a hang.
struct GridBar {
    unsigned count, gen;
    int err, pad;
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_relaxed_gpu(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// True when every one of `expect` CTAs has arrived; false when the wait ran
// out or another CTA's did.  Memory written by any thread of any CTA before
// the barrier is visible to every thread after it.
__device__ __forceinline__ bool grid_sync(GridBar* b, unsigned expect, unsigned long long limit_ns) {
    if (expect == 1) {   // a grid of one CTA: the block barrier orders its global memory as well
        __syncthreads();
        return true;
    }
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        const unsigned g = ld_acquire_gpu(&b->gen);
        __threadfence();   // the CTA's writes, ordered by the barrier above, before the arrival
        if (atom_add_acq_rel_gpu(&b->count, 1u) == expect - 1) {
            atomicExch(&b->count, 0u);
            st_release_gpu(&b->gen, g + 1);
        } else {
            const unsigned long long t0 = globaltimer_ns();
            while (ld_acquire_gpu(&b->gen) == g) {
                if (ld_relaxed_gpu(&b->err) || globaltimer_ns() - t0 > limit_ns) {
                    atomicExch(&b->err, 1);
                    good = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// Arithmetic with its rounding fixed.  The compiler may fuse a multiply and an
// add of a plain expression differently in different kernels (which of two
// products to fuse, a select of products, a product by two turned into an
// add); rmul never fuses and rfma always does, so a step written with them
// gives the same bits in every kernel that runs it.
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return __fma_rn(a, b, c); }

// ---- the checked build ----------------------------------------------------
// Built with RB200_DEBUG_BOUNDS (python -m reformulation_b200.build
// --debug-bounds, a library of its own), every gather and scatter whose index
// comes from data is checked: index_ok() returns false for an index out of
// range, marks the solver's control block (status = kBoundsStatus; the run
// returns an error) and the caller skips the access, so a bad index is
// reported instead of read or written.  In the normal build index_ok() is
// `true` and costs nothing.
#ifdef RB200_DEBUG_BOUNDS
constexpr bool kDebugBounds = true;
#else
constexpr bool kDebugBounds = false;
#endif
constexpr int kBoundsStatus = 2;

__device__ __forceinline__ bool index_ok(bool ok, int* status) {
    if constexpr (kDebugBounds) {
        if (!ok) atomicExch(status, kBoundsStatus);
        return ok;
    } else {
        return true;
    }
}

// The convergence trace: a ring of `cap` records (reform_trace_record,
// include/reform_trace.h) in device memory, `len` written so far; the next
// goes to len % cap.  Written by the one thread that takes a check's
// decisions, so no ordering beyond the check's own is needed.
__device__ __forceinline__ void trace_put(reform_trace_record* ring, int cap, long long& len, long long iteration,
                                          double gap, double error, double omega, double lower, double upper,
                                          int restart, int terminated) {
    if (!ring || cap <= 0) return;
    reform_trace_record& r = ring[len % cap];
    r.iteration = iteration;
    r.gap = gap;
    r.error = error;
    r.omega = omega;
    r.lower = lower;
    r.upper = upper;
    r.restart = restart;
    r.terminated = terminated;
    ++len;
}

template <class T>
__device__ __forceinline__ T clampv(T v, T lo, T hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

inline int ceil_div(long long a, long long b) { return int((a + b - 1) / b); }

// A fact the set-up asks the driver for (an occupancy, a kernel attribute, a
// device attribute), asked once per process and device and then remembered:
// `query(int*)` runs the first time for the current device.  Each call site
// passes its own lambda, whose type keys the memo.
template <class Query>
cudaError_t once_per_device(int* out, Query query) {
    static std::mutex mu;
    static int value[64];
    static bool known[64] = {};
    int dev = 0;
    RB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!known[dev]) {
        RB_CUDA_TRY(query(&value[dev]));
        known[dev] = true;
    }
    *out = value[dev];
    return cudaSuccess;
}

}  // namespace rb200
