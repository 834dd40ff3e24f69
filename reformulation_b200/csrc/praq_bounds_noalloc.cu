// praq_bounds_noalloc.cu -- the roof-dual bracket of a given primal-dual pair,
// computed on the caller's stream with no device allocation at all.
//
// Why it exists: some callers cannot allocate device memory at the point where
// they want a certificate -- code that runs inside its own stream capture
// (allocation calls are not capturable), real-time loops whose policy forbids
// the allocator, and hosts such as frameworks that own every byte of device
// memory and give a library only the buffers it is handed.  They hold the
// instance, the point and a two-double output in memory they allocated
// themselves; this entry point keeps its own scratch (the per-node Sᵀy
// accumulator and the per-block partial sums) in one file-scope __device__
// array of fixed size instead of asking for any.
//
// What it computes is the bracket of qubo/praq-jax/praq/solver.py:320-362
// (relaxation_bounds), in the instance's own units:
//   upper = sum_i d_i x_i + sum_e [W_e > 0 ? 2W_e max(x_i + x_j - 1, 0)
//                                          : 2W_e min(x_i, x_j)]
//   lower = sum_i min(d_i - (S^T y)_i, 0) + sum over covering edges of y_e,1
// for x in [0, 1]^n and half-edge duals y (pairs, instance units).
#include "../../include/praq.h"
#include "common.cuh"

#include <mutex>

namespace rb200 {
namespace noalloc {

// The maximum instance this entry point takes, and its scratch layout:
//   [0, kMaxNodes)                       the S^T y accumulator
//   [kMaxNodes, kMaxNodes + 4 kBlocks)   two partial rows (upper, lower) per
//                                        block, for the edge pass then the
//                                        node pass
//   [kMaxNodes + 4 kBlocks]              a flag: an edge index was out of
//                                        range, or an edge was a self-loop
constexpr long long kMaxNodes = 1LL << 18;   // 262,144 nodes: 2 MiB of doubles
constexpr int kBlocks = 296;                 // fixed grid: 2 blocks per SM on 148 SMs
constexpr int kThreads = 256;
constexpr long long kScratchDoubles = kMaxNodes + 4 * kBlocks + 1;

// Shared by every call on this device; holds the last call's contents.
static __device__ __align__(256) double g_scratch[kScratchDoubles];

__global__ void clear_kernel(long long n, double* __restrict__ s) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) s[i] = 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) s[kMaxNodes + 4 * kBlocks] = 0.0;
}

// Edge pass: accumulate both half-edge duals into S^T y (FP64 atomics, so
// the order of the additions into one node, and with it the last bits of the
// lower bound, can change from call to call), and the edge parts of both
// bounds into this block's partial row.
__global__ void __launch_bounds__(kThreads)
edge_pass(long long n, long long m, const int64_t* __restrict__ rows, const int64_t* __restrict__ cols,
          const double* __restrict__ vals, const double* __restrict__ x, const double* __restrict__ y,
          double* __restrict__ s) {
    __shared__ double scratch[2 * 32];
    double acc[2] = {0.0, 0.0};
    bool bad = false;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
        const int64_t i = rows[e], j = cols[e];
        if (i < 0 || i >= n || j < 0 || j >= n || i == j) {   // out of range or a self-loop
            bad = true;
            continue;
        }
        const double w = 2.0 * vals[e], y0 = y[2 * e], y1 = y[2 * e + 1];
        const double xi = x[i], xj = x[j];
        atomicAdd(&s[i], y0);
        atomicAdd(&s[j], y1);
        acc[0] += w > 0.0 ? w * fmax(xi + xj - 1.0, 0.0) : w * fmin(xi, xj);
        acc[1] += w > 0.0 ? y0 : 0.0;
    }
    if (bad) s[kMaxNodes + 4 * kBlocks] = 1.0;
    block_sums<2>(acc, scratch, acc);
    if (threadIdx.x == 0) {
        s[kMaxNodes + 2 * blockIdx.x] = acc[0];
        s[kMaxNodes + 2 * blockIdx.x + 1] = acc[1];
    }
}

// Node pass: the node parts of both bounds into the second set of rows.
__global__ void __launch_bounds__(kThreads)
node_pass(long long n, const double* __restrict__ diag, const double* __restrict__ x, double* __restrict__ s) {
    __shared__ double scratch[2 * 32];
    double acc[2] = {0.0, 0.0};
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double d = diag[i];
        acc[0] += d * x[i];
        const double rc = d - s[i];
        acc[1] += rc < 0.0 ? rc : 0.0;
    }
    block_sums<2>(acc, scratch, acc);
    if (threadIdx.x == 0) {
        s[kMaxNodes + 2 * kBlocks + 2 * blockIdx.x] = acc[0];
        s[kMaxNodes + 2 * kBlocks + 2 * blockIdx.x + 1] = acc[1];
    }
}

// One block: both sets of partial rows, in a fixed order, into out[0] (lower)
// and out[1] (upper); NaN for both if an edge was out of range or a self-loop.
__global__ void __launch_bounds__(kThreads) finish(const double* __restrict__ s, double* __restrict__ out) {
    __shared__ double scratch[2 * 32];
    __shared__ double total[2];
    reduce_rows<2>(s + kMaxNodes, 2 * kBlocks, scratch, total);
    if (threadIdx.x == 0) {
        const bool bad = s[kMaxNodes + 4 * kBlocks] != 0.0;
        out[0] = bad ? NAN : total[1];
        out[1] = bad ? NAN : total[0];
    }
}

// The device address of g_scratch, looked up once per device (with that
// device current) and cached for the life of the process: a cudaDeviceReset
// unloads the module and leaves the cached address stale.
static double* scratch_address() {
    static std::mutex mu;
    static double* cache[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!cache[dev]) {
        double* p = nullptr;
        if (cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_scratch) != cudaSuccess) return nullptr;
        cache[dev] = p;
    }
    return cache[dev];
}

}  // namespace noalloc
}  // namespace rb200

extern "C" int reform_praq_bounds_noalloc(int64_t n, int64_t m, const double* diag,
                                          const int64_t* rows, const int64_t* cols,
                                          const double* vals, const double* x, const double* y,
                                          double* out, void* stream) {
    using namespace rb200::noalloc;
    if (!diag || !x || !out || (m > 0 && (!rows || !cols || !vals || !y))) return PRAQ_ERROR_ARGUMENT;
    if (n <= 0 || n > kMaxNodes || m < 0) return PRAQ_ERROR_INSTANCE;
    // An error the caller left pending on this thread is reported, not
    // cleared, and nothing is launched; after that check every error of the
    // launches below is this call's own.
    if (cudaPeekAtLastError() != cudaSuccess) return PRAQ_ERROR_CUDA;
    double* s = scratch_address();
    if (!s) return PRAQ_ERROR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    clear_kernel<<<kBlocks, kThreads, 0, st>>>(n, s);
    if (cudaGetLastError() != cudaSuccess) return PRAQ_ERROR_CUDA;
    edge_pass<<<kBlocks, kThreads, 0, st>>>(n, m, rows, cols, vals, x, y, s);
    if (cudaGetLastError() != cudaSuccess) return PRAQ_ERROR_CUDA;
    node_pass<<<kBlocks, kThreads, 0, st>>>(n, diag, x, s);
    if (cudaGetLastError() != cudaSuccess) return PRAQ_ERROR_CUDA;
    finish<<<1, kThreads, 0, st>>>(s, out);
    return cudaGetLastError() == cudaSuccess ? 0 : PRAQ_ERROR_CUDA;
}
