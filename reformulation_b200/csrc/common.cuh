// common.cuh -- shared device/host helpers for the PRAQ and PRIA solvers.
//
// Everything here is plain sm_100a CUDA C++: warp shuffles, shared memory and
// fixed-order block reductions (deterministic: the order of additions depends
// on the launch shape only, so a solve is bitwise reproducible run to run).
#pragma once

#include <utility>

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <limits>
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

template <class T>
__device__ __forceinline__ T clampv(T v, T lo, T hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

inline int ceil_div(long long a, long long b) { return int((a + b - 1) / b); }

}  // namespace rb200
