// pria_core.cuh -- PRIA (the joint replenishment LP) on B200: restarted,
// reflected Halpern PDHG on upper-triangular simplices, FP64 or FP32 iterates
// with FP64 reductions, restart logic and bounds.
//
// The algorithm is the reference's (jrp/pria-jax/pria/solver.py, the
// specification; jrp/pria-cuda/src/*.cuh, its CUDA port):
//     x' = P_X(x - tau (h + y + z))         per (i, t): the column s <= t onto
//                                           the unit simplex
//     r  = sigma (2 x' - x)
//     y' = P_Y(y + r)                       per (i, s): the row t >= s onto the
//                                           K_i simplex
//     z' = P_Z(z + r)                       per s: the group {(i, t >= s)} onto
//                                           the K0 simplex
// with the Halpern combination, the canonical norm with a NEGATIVE cross term
// (halpern_operator.py:5-19), the bounds of solver.py:347-402 and the restart
// logic of solver.py:514-594.
//
// Device design (this file's own):
// * PERIOD-MAJOR PACKED TRIANGLE.  Entry (i, s, t), s <= t < Tp, lives at
//   blk(s) + i (Tp - s) + (t - s), blk(s) = N (s Tp - s (s - 1) / 2): block s
//   holds every item's row s.  A y row is contiguous, a z group is one
//   contiguous block, and an x column is one short run per block.
// * x HALF-STEP: one CTA per (item, tile of TW columns), heaviest tiles first.
//   It reads the tile's row runs coalesced (TW consecutive periods per row),
//   forms pre = x - tau (h + y + z) in a shared-memory tile stored column-major
//   with an odd column stride (bank-conflict free for the column passes), runs
//   one warp-level Michelot projection per column (theta <- (sum_{v>theta} v -
//   1) / #{v > theta} to the fixed point, warp-shuffle sums), and writes the
//   reflection r and the next step's combined x.
// * y/z HALF-STEP: one thread-block CLUSTER per period block s.  Each warp
//   projects y rows held in registers (Michelot, shuffles); the block's z
//   values sit in the CTAs' shared memory and the z Michelot runs across the
//   cluster, each round exchanging (sum, count) through distributed shared
//   memory.  r is read once for both.
// * x, y, z hold the NEXT step's Halpern-combined point (as PRAQ's dual), so a
//   reflected step streams x, x0, h, y, z (x kernel) and y, y0, z, z0, r (y/z
//   kernel) and writes x, r, y, z: 14 ND reals per iteration.
// * Decisions on the device (check_kernel); a block of op_steps steps plus
//   the gated restart step replays as a captured CUDA graph.
#pragma once

#include "../../include/pria.h"
#include "common.cuh"
#include "memory.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <memory>

namespace cg = cooperative_groups;

namespace rb200 {
namespace pria {
namespace {

constexpr int kMaxPeriods = 1024;       // padded periods (a y row lives in 32 registers per lane)
constexpr int kXThreads = 256;
constexpr int kAuxThreads = 256;
constexpr int kCheckBlock = 256;
constexpr int kLowTW = 32;              // columns per tile of the lower-bound pass
#ifndef RB200_PRIA_XTILE
#define RB200_PRIA_XTILE 8              // compile-time tunable (sweeps build with -D)
#endif
constexpr int kXTile = RB200_PRIA_XTILE;   // columns per tile of the x half-step (FP64 tile)
// z half-step CTA: threads and the shared-memory slice of a period block it
// holds, per precision (compile-time tunables; sweeps build with -D).
// Measured per solve (PRIA N = 100, T = 500 / N = 200, T = 300 / N = 60,
// T = 200): FP64 with 256 threads 46.5 / 35.9 / 6.0 ms against 52.6 / 39.2 /
// 5.9 with 512; FP32 with 512 threads and 96 KB slices 32.3 / 27.2 / 5.3 ms
// (256 threads and 48 KB: 31.8 / 26.4 / 5.7).
#ifndef RB200_PRIA_ZSLICE_KB
#define RB200_PRIA_ZSLICE_KB 96
#endif
#ifndef RB200_PRIA_ZSLICE_KB_F64
#define RB200_PRIA_ZSLICE_KB_F64 96
#endif
constexpr int kMaxCluster = 16;
// rows per warp in flight (x kernel): 6 in FP32, 4 in FP64 (measured best
// of 2, 3, 4, 6, 8 for each; 6 in FP64 and 8 in either hold too many registers)
template <class Real>
constexpr int x_unroll() { return sizeof(Real) == 4 ? 6 : 4; }
constexpr int kZUnroll = 8;          // z elements per thread in flight (z kernel)
// y row values per lane in flight (y kernel): 8 in FP32, 4 in FP64 (more
// registers per value; measured best of 4, 8, 16 for each)
template <class Real>
constexpr int y_chunk() { return sizeof(Real) == 4 ? 8 : 4; }
constexpr int kYThreads = 256;       // y kernel: one warp per row, kYThreads / 32 rows per tile
#ifndef RB200_PRIA_ZTHREADS
#define RB200_PRIA_ZTHREADS 512
#endif
#ifndef RB200_PRIA_ZTHREADS_F64
#define RB200_PRIA_ZTHREADS_F64 256
#endif
template <class Real>
constexpr int z_threads() { return sizeof(Real) == 8 ? RB200_PRIA_ZTHREADS_F64 : RB200_PRIA_ZTHREADS; }
template <class Real>
constexpr int z_slice_bytes() {
    return (sizeof(Real) == 8 ? RB200_PRIA_ZSLICE_KB_F64 : RB200_PRIA_ZSLICE_KB) * 1024;
}

struct Control {
    double omega, theta, fp_error, check_error;
    double new_error, lower, upper, gap;
    long long restart_iter, iteration;
    int terminated, restart, result_slot, status;
    int phase_done;          // the vanilla phase reached its step budget
    long long trace_len;     // convergence-trace records written this run
};

struct Params {
    double tolerance, eta;
    long long max_iter, op_steps;
    double beta_sufficient, beta_necessary, beta_artificial;
    double theta_target, theta_decay;
    double scale;
    long long start_max;     // step budget the start check compares against
    long long vanilla_max;   // step budget of the vanilla phase (< 0: none)
    double omega0;           // the initial primal weight
    int vanilla_solve;       // plain PDHG throughout (no Halpern phase)
    reform_trace_record* trace;   // the convergence-trace ring (null: none)
    int trace_cap;
};

// Bits of the `gate` argument of the step kernels.
constexpr int kGateRestart = 1;   // run only when the last check asked for a restart
constexpr int kGateVanilla = 2;   // vanilla step: next point = the step, anchor untouched
constexpr int kGateDrift = 4;     // check sums measure the drift from the existing anchor

__host__ __device__ __forceinline__ long long blk(int n, int tp, int s) {
    return (long long)n * ((long long)s * tp - (long long)s * (s - 1) / 2);
}

template <class Real>
struct alignas(16) Dev {   // (16-byte aligned: the batched engine copies descriptors in 16-byte pieces)
    int n, t, tp, ntc, ntc_low, csize;
    int zpair;               // 1: the solver's z launch takes period blocks in pairs (s, Tp - 1 - s)
                             //    (z_task_pair); 0: one block per cluster (z_task, which the
                             //    batched engine always uses; the slice fits either way)
    int zstaged;             // 1: z + r of a task sits in its cluster's shared memory;
                             // 0: too large for that, every Michelot round recomputes
                             //    it from global memory (L2-resident)
    long long nd;
    double eta;
    const Real* h;           // [nd] holding costs / scale
    const Real* k;           // [n] K_i / scale
    Real k0;                 // K0 / scale
    Real *xh, *x0, *r, *yh, *y0, *zh, *z0;   // combined point (next step), anchors, reflection
    Real *x2s, *dxs, *y2s, *z2s;             // at checks: the step and x1 - x2
    double *px, *py, *pyz, *pup, *plo;       // partial rows (pyz: the z half-step's)
    double *thx, *thy, *thz;                 // last thresholds: per column, row, block
    Control* ctl;
};

__device__ __forceinline__ bool skip(const Control* c, int gate) {
    return c->terminated || ((gate & kGateRestart) && !c->restart);
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Michelot's simplex projection threshold: theta with
// sum max(v - theta, 0) = target, the fixed point of
//     theta <- (sum_{v > theta} v - target) / #{v > theta}.
// From the all-active start the active count falls strictly until the fixed
// point.  A warm start (the segment's threshold of the previous iteration,
// which moves little from one iteration to the next) takes the active set at
// `warm`; the first update from it lands at or below the fixed point whatever
// side `warm` was on, and from there the count falls again.  When the count
// stops falling in that monotone phase the loop ends: rounding can move theta
// back by an ulp and let an element re-enter, which would otherwise cycle.
// A warm start with an empty active set falls back to the cold start.
// Returns +inf for target <= 0 (the zero simplex).

// sums over {v > th} for values held by one warp in registers
template <class Real, int K>
__device__ __forceinline__ void active_regs(const Real (&v)[K], int len, double th, double& S, int& C) {
    const int lane = threadIdx.x & 31;
    const Real thr = Real(th);
    Real p = Real(0);
    int c = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (lane + 32 * k < len && (th == -INFINITY || v[k] > thr)) {
            p += v[k];
            ++c;
        }
    }
    S = warp_sum(double(p));
    C = __reduce_add_sync(0xffffffffu, c);
}

template <class Real>
__device__ __forceinline__ void active_smem(const Real* v, int len, double th, double& S, int& C) {
    const int lane = threadIdx.x & 31;
    double p = 0.0;
    int c = 0;
    for (int q = lane; q < len; q += 32) {
        const double x = double(v[q]);
        if (th == -INFINITY || x > th) {
            p += x;
            ++c;
        }
    }
    S = warp_sum(p);
    C = __reduce_add_sync(0xffffffffu, c);
}

// The Michelot iteration over an `active(th, S, C)` sum routine; `warm` is
// NaN for a cold start.
template <class F>
__device__ __forceinline__ double michelot(F active, int len, double target, double warm) {
    if (!(target > 0.0)) return INFINITY;
    double S;
    int C;
    bool monotone = true;
    if (isfinite(warm)) {
        active(warm, S, C);
        monotone = false;
    }
    if (!isfinite(warm) || C == 0) {
        active(-INFINITY, S, C);   // all active
        monotone = true;
    }
    double th = (S - target) / double(C);
    for (int round = 0; round <= len; ++round) {
        double S2;
        int C2;
        active(th, S2, C2);
        if (C2 == C || C2 == 0) break;
        if (monotone && C2 > C) break;
        monotone = true;
        S = S2;
        C = C2;
        th = (S2 - target) / double(C2);
    }
    return th;
}

template <class Real, int K>
__device__ double michelot_regs(const Real (&v)[K], int len, double target, double warm) {
    return michelot([&](double th, double& S, int& C) { active_regs(v, len, th, S, C); }, len, target,
                    warm);
}

template <class Real>
__device__ double michelot_smem(const Real* v, int len, double target, double warm) {
    return michelot([&](double th, double& S, int& C) { active_smem(v, len, th, S, C); }, len, target,
                    warm);
}

// x half-step of one PDHG step (solver.py:418-421), with the reflection and
// the next combined x.  Reflect: the point stepped from is xsrc (= xh);
// vanilla: xsrc is the point itself and becomes the anchor.  Check: x2 and
// x1 - x2 are kept and the x sums go to px.
template <class Real, int TW, bool Reflect, bool Check>
__device__ __forceinline__ void x_kernel_tile(const Dev<Real>& d, int tile, const Real* xsrc, const Real* ysrc, const Real* zsrc,
         int step, int gate) {
    const Control* c = d.ctl;
    if (skip(c, gate)) return;
    // The tile of pre = x - tau (h + y + z) is FP64 whatever Real is: tau h
    // can exceed x by many orders of magnitude (the duals' scale is K / scale
    // per entry, the primal's is 1), and the column threshold cancels that
    // common part, so pre must carry the digits FP32 would drop.
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* pre = reinterpret_cast<double*>(smem_raw);
    __shared__ double theta[TW];
    __shared__ double scratch[2 * 32];
    const int item = tile % d.n;
    const int ctile = d.ntc - 1 - int(tile / d.n);   // heaviest tiles first
    const int t0 = ctile * TW;
    const int tcols = min(TW, d.tp - t0);
    const int rows = t0 + tcols;
    const int stride = rows | 1;
    constexpr int kRpw = 32 / TW;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int col = lane % TW, sub = lane / TW;
    const int tt = t0 + col;
    const double om = c->omega;
    const double tau = d.eta / om, sigma = d.eta * om;
    constexpr int kUnroll = x_unroll<Real>();
    // rows are taken kUnroll at a time per warp so that their loads are in
    // flight together
    const int rstep = nwarps * kRpw;
    for (int sb = warp * kRpw + sub; sb < rows; sb += rstep * kUnroll) {
        long long ev[kUnroll];
        Real xv[kUnroll], hv[kUnroll], yv[kUnroll], zv[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const int s = sb + u * rstep;
            ev[u] = -1;
            if (s < rows && col < tcols && tt >= s &&
                index_ok(blk(d.n, d.tp, s) + (long long)item * (d.tp - s) + (tt - s) < d.nd, &d.ctl->status)) {
                ev[u] = blk(d.n, d.tp, s) + (long long)item * (d.tp - s) + (tt - s);
                xv[u] = xsrc[ev[u]];
                hv[u] = d.h[ev[u]];
                yv[u] = ysrc[ev[u]];
                zv[u] = zsrc[ev[u]];
                // the anchor the second pass reads, on chip by then
                if ((Reflect || (gate & kGateDrift)) && ((col & 7) == 0 || tt == s)) prefetch_l2(d.x0 + ev[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u)
            if (ev[u] >= 0)
                pre[col * stride + sb + u * rstep] =
                    double(xv[u]) - tau * ((double(hv[u]) + double(yv[u])) + double(zv[u]));
    }
    __syncthreads();
    for (int cc = warp; cc < tcols; cc += nwarps) {
        double* slot = d.thx + (long long)item * d.tp + (t0 + cc);
        const double th = michelot_smem(pre + cc * stride, t0 + cc + 1, 1.0, *slot);
        if (lane == 0) {
            theta[cc] = th;
            *slot = th;
        }
    }
    __syncthreads();
    const double kn = Reflect ? double(c->restart_iter + step + 2) : 1.0;
    const double lwn = kn / (kn + 1.0), rwn = 1.0 / (kn + 1.0);
    // Without Reflect: a vanilla step (the next point is the step itself and
    // the anchor stays), or the step that makes the point stepped from the
    // new anchor (restart; the end of the vanilla phase, whose drift sums are
    // taken against the old anchor).
    const bool vanilla = !Reflect && (gate & kGateVanilla);
    const bool drift = Reflect || (gate & kGateDrift);
    double acc[2] = {0.0, 0.0};
    for (int sb = warp * kRpw + sub; sb < rows; sb += rstep * kUnroll) {
        long long ev[kUnroll];
        Real x1v[kUnroll], xav[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const int s = sb + u * rstep;
            ev[u] = -1;
            if (s < rows && col < tcols && tt >= s &&
                index_ok(blk(d.n, d.tp, s) + (long long)item * (d.tp - s) + (tt - s) < d.nd, &d.ctl->status)) {
                ev[u] = blk(d.n, d.tp, s) + (long long)item * (d.tp - s) + (tt - s);
                x1v[u] = xsrc[ev[u]];
                xav[u] = drift ? d.x0[ev[u]] : x1v[u];
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            if (ev[u] < 0) continue;
            const long long e = ev[u];
            const Real x2 = Real(fmax(pre[col * stride + sb + u * rstep] - theta[col], 0.0));
            const Real x1 = x1v[u], xa = Reflect ? xav[u] : x1;
            const double refl = 2.0 * double(x2) - double(x1);
            d.r[e] = Real(sigma * refl);
            d.xh[e] = vanilla ? x2 : Real(lwn * refl + rwn * double(xa));
            if (!Reflect && !vanilla) d.x0[e] = x1;
            if (Check) {
                d.x2s[e] = x2;
                d.dxs[e] = x1 - x2;
                const double dx = double(x1) - double(x2), dr = double(x1) - double(xav[u]);
                acc[0] += dx * dx;
                acc[1] += dr * dr;
            }
        }
    }
    if (Check) {
        block_sums<2>(acc, scratch, acc);
        if (threadIdx.x == 0) {
            d.px[size_t(tile) * 2] = acc[0];
            d.px[size_t(tile) * 2 + 1] = acc[1];
        }
    }
}

template <class Real, int TW, bool Reflect, bool Check>
__global__ void __launch_bounds__(kXThreads)
x_kernel(Dev<Real> d, const Real* xsrc, const Real* __restrict__ ysrc, const Real* __restrict__ zsrc,
         int step, int gate) {
    x_kernel_tile<Real, TW, Reflect, Check>(d, blockIdx.x, xsrc, ysrc, zsrc, step, gate);
}

// y half-step (solver.py:421-422) for one tile of rows: warp w takes row
// g = tile * (rows per tile) + w of the period-major order (block s, item i),
// a contiguous run of Tp - s values.  y' = P_Y(y + r) onto the K_i simplex
// (Michelot over the row staged in the warp's slice of shared memory,
// warm-started from the row's last threshold), the next combined y, and at
// checks y2 and the y parts of the check sums.  `rows` holds
// (threads / 32) * row_cap reals, row_cap >= Tp.
template <class Real, bool Reflect, bool Check>
__device__ __forceinline__ void y_kernel_tile(const Dev<Real>& d, int tile, const Real* ysrc, int step, int gate,
                                              Real* rows, int row_cap) {
    const Control* c = d.ctl;
    if (skip(c, gate)) return;
    __shared__ double scratch[3 * 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Real* v = rows + size_t(warp) * row_cap;
    const long long g = (long long)tile * (blockDim.x >> 5) + warp;
    const double kn = Reflect ? double(c->restart_iter + step + 2) : 1.0;
    const Real lwn = Real(kn / (kn + 1.0)), rwn = Real(1.0 / (kn + 1.0));
    // Without Reflect: a vanilla step (next = the step, anchor kept) or the
    // step that makes the current point the anchor (drift against the old one)
    const bool vanilla = !Reflect && (gate & kGateVanilla);
    const bool drift = Reflect || (gate & kGateDrift);
    double acc[3] = {0.0, 0.0, 0.0};   // |dy|^2, <dx, dy>, drift
    constexpr int kYChunk = y_chunk<Real>();
    if (g < (long long)d.tp * d.n) {    // uniform over the warp
        const int s = int(g / d.n), i = int(g - (long long)s * d.n);
        const int len = index_ok(blk(d.n, d.tp, s) + (long long)(i + 1) * (d.tp - s) <= d.nd, &d.ctl->status)
                            ? d.tp - s : 0;
        const long long e0 = blk(d.n, d.tp, s) + (long long)i * (d.tp - s);
        // chunks of kYChunk values per lane, loaded by predicated loads with
        // no loop around them, so each chunk is one memory round trip (an
        // unrolled loop over the row would end in a remainder loop that waits
        // for every load in turn)
        for (int q0 = 0; q0 < len; q0 += 32 * kYChunk) {   // uniform over the warp
            Real a[kYChunk], b[kYChunk];
#pragma unroll
            for (int u = 0; u < kYChunk; ++u) {
                const int q = q0 + lane + 32 * u;
                if (q < len) {
                    a[u] = ysrc[e0 + q];
                    b[u] = d.r[e0 + q];
                    if (drift && (q & 7) == 0) prefetch_l2(d.y0 + e0 + q);   // one per 32-byte sector
                    if (Check && (q & 7) == 0) prefetch_l2(d.dxs + e0 + q);
                }
            }
#pragma unroll
            for (int u = 0; u < kYChunk; ++u) {
                const int q = q0 + lane + 32 * u;
                if (q < len) v[q] = a[u] + b[u];
            }
        }
        __syncwarp();
        double* slot = d.thy + (long long)s * d.n + i;
        const double th = michelot_smem(v, len, double(d.k[i]), *slot);
        if (lane == 0) *slot = th;
        for (int q0 = 0; q0 < len; q0 += 32 * kYChunk) {   // uniform over the warp
            Real y1v[kYChunk], ydv[kYChunk], dxv[kYChunk];
#pragma unroll
            for (int u = 0; u < kYChunk; ++u) {
                const int q = q0 + lane + 32 * u;
                if (q < len) {
                    y1v[u] = ysrc[e0 + q];
                    ydv[u] = drift ? d.y0[e0 + q] : y1v[u];
                    if (Check) dxv[u] = d.dxs[e0 + q];
                }
            }
#pragma unroll
            for (int u = 0; u < kYChunk; ++u) {
                const int q = q0 + lane + 32 * u;
                if (q >= len) continue;
                const long long e = e0 + q;
                const Real y2 = Real(fmax(double(v[q]) - th, 0.0));
                const Real y1 = y1v[u], yd = ydv[u];
                const Real ya = Reflect ? yd : y1;
                d.yh[e] = vanilla ? y2 : lwn * (Real(2) * y2 - y1) + rwn * ya;
                if (!Reflect && !vanilla) d.y0[e] = y1;
                if (Check) {
                    if (Reflect) d.y2s[e] = y2;
                    const double dy = double(y1) - double(y2), dr = double(y1) - double(yd);
                    acc[0] += dy * dy;
                    acc[1] += double(dxv[u]) * dy;
                    acc[2] += dr * dr;
                }
            }
        }
    }
    if (Check) {
        block_sums<3>(acc, scratch, acc);
        if (threadIdx.x == 0)
            for (int k = 0; k < 3; ++k) d.py[size_t(tile) * 3 + k] = acc[k];
    }
}

template <class Real, bool Reflect, bool Check>
__global__ void __launch_bounds__(kYThreads)
y_kernel(Dev<Real> d, const Real* ysrc, int step, int gate) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    y_kernel_tile<Real, Reflect, Check>(d, blockIdx.x, ysrc, step, gate, reinterpret_cast<Real*>(smem_raw), d.tp);
}

// michelot() advanced one evaluation at a time, so that several problems can
// share each (cluster-wide) evaluation: init, then while !done() evaluate the
// sums (S, C) over {v > th} (all v when th is -inf) and feed() them.  The
// steps and decisions are michelot()'s, one for one; th is the result once
// done().
struct MichelotSteps {
    double target, th, S;
    int C, len, round, stage;   // stage 0: warm pending, 1: all-active pending, 2: round pending, 3: done
    bool monotone;
    __device__ __forceinline__ void init(double tgt, double warm, int n_) {
        target = tgt;
        len = n_;
        round = 0;
        S = 0.0;
        C = 0;
        monotone = true;
        if (!(tgt > 0.0)) {
            th = INFINITY;
            stage = 3;
        } else if (isfinite(warm)) {
            th = warm;
            stage = 0;
        } else {
            th = -INFINITY;
            stage = 1;
        }
    }
    __device__ __forceinline__ bool done() const { return stage == 3; }
    __device__ __forceinline__ void feed(double S2, int C2) {
        if (stage == 0) {
            S = S2;
            C = C2;
            monotone = false;
            if (C == 0) {
                th = -INFINITY;
                stage = 1;
            } else {
                th = (S - target) / double(C);
                stage = 2;
            }
        } else if (stage == 1) {
            S = S2;
            C = C2;
            monotone = true;
            th = (S - target) / double(C);
            stage = 2;
        } else if (stage == 2) {
            if (C2 == C || C2 == 0 || (monotone && C2 > C)) {
                stage = 3;
                return;
            }
            monotone = true;
            S = S2;
            C = C2;
            th = (S2 - target) / double(C2);
            if (++round > len) stage = 3;
        }
    }
};

// The CTAs that share one z task: the CTAs of a cluster (ZGroup<false>), or
// one CTA alone (ZGroup<true>, the persistent kernel, whose launch has no
// clusters), with the same interface so that z_task's arithmetic is one code.
template <bool Solo>
struct ZGroup {
    cg::cluster_group g = cg::this_cluster();
    __device__ __forceinline__ int rank() const { return int(g.block_rank()); }
    __device__ __forceinline__ void sync() { g.sync(); }
    template <class T>
    __device__ __forceinline__ T* peer(T* p, int r) { return g.map_shared_rank(p, r); }
};
template <>
struct ZGroup<true> {
    __device__ __forceinline__ int rank() const { return 0; }
    __device__ __forceinline__ void sync() { __syncthreads(); }
    template <class T>
    __device__ __forceinline__ T* peer(T* p, int) { return p; }
};

// Sums of K values over every thread of every CTA of a cluster, bitwise the
// same on every CTA, with one cluster barrier: each warp's total goes to its
// slot of slots[parity]; after the barrier warp 0 of each CTA adds all ranks'
// slots (lane l takes slots l, l + 32, ... in order, then a shuffle tree, the
// same on every CTA) and one CTA barrier hands the totals to every thread.
// A round may reuse slots[parity] two rounds later: the barrier of the round
// between them is reached by every warp 0 only after its reads.
template <int K, int kWarps, class Group>
__device__ __forceinline__ void cluster_sums(const double (&v)[K], double (*slots)[kWarps][K], double* tot,
                                             int parity, Group& cluster, int csize, double (&out)[K]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const double w = warp_sum(v[k]);
        if (lane == 0) slots[parity][warp][k] = w;
    }
    cluster.sync();
    if (warp == 0) {
        double a[K];
#pragma unroll
        for (int k = 0; k < K; ++k) a[k] = 0.0;
        for (int idx = lane; idx < csize * kWarps; idx += 32) {
            const double* pp = cluster.peer(&slots[parity][idx % kWarps][0], idx / kWarps);
#pragma unroll
            for (int k = 0; k < K; ++k) a[k] += pp[k];
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            a[k] = warp_sum(a[k]);
            if (lane == 0) tot[parity * K + k] = a[k];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = tot[parity * K + k];
}

// z half-step (solver.py:423) for period block s, one cluster of `csize` CTAs
// per block; CTA `rank` owns rows [r0, r1) of the block, a contiguous slice.
// z + r of the slice goes to shared memory, the threshold of the whole block
// comes from Michelot rounds whose (sum, count) pass through distributed
// shared memory, then the slice's z is written.  Solo: the whole block in
// this CTA (csize 1), CTA barriers in place of cluster barriers, the same
// sums in the same order.
template <class Real, int kThreads, bool Reflect, bool Check, bool Solo = false>
__device__ __forceinline__ void z_task(const Dev<Real>& d, int s, const Real* zsrc, int step, int gate) {
    const Control* c = d.ctl;
    if (skip(c, gate)) return;   // uniform over the cluster: c is not written here
    ZGroup<Solo> cluster;
    const int csize = Solo ? 1 : d.csize;
    const int rank = cluster.rank();
    const int len = d.tp - s;
    const long long base = blk(d.n, d.tp, s);
    const int r0 = int((long long)d.n * rank / csize), r1 = int((long long)d.n * (rank + 1) / csize);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real* vz = reinterpret_cast<Real*>(smem_raw);
    __shared__ double slots[2][kThreads / 32][2];
    __shared__ double tot[2 * 2];
    __shared__ double scratch[3 * 32];
    const double kn = Reflect ? double(c->restart_iter + step + 2) : 1.0;
    const Real lwn = Real(kn / (kn + 1.0)), rwn = Real(1.0 / (kn + 1.0));
    const bool vanilla = !Reflect && (gate & kGateVanilla);   // as in the y half-step
    const bool drift = Reflect || (gate & kGateDrift);
    double acc[3] = {0.0, 0.0, 0.0};   // |dz|^2, <dx, dz>, drift
    const long long sbase = base + (long long)r0 * len;
    const int mine = index_ok(sbase + (long long)(r1 - r0) * len <= d.nd, &d.ctl->status) ? (r1 - r0) * len : 0;

    const bool staged = d.zstaged != 0;
    // v(q) = z + r of the slice's element q, in the same arithmetic either way
    auto vval = [&](int q) -> Real { return staged ? vz[q] : Real(zsrc[sbase + q] + d.r[sbase + q]); };

    // phase A: z + r of the slice into shared memory, kZUnroll loads in flight
    for (int qb = threadIdx.x; staged && qb < mine; qb += kThreads * kZUnroll) {
        Real zv[kZUnroll], rv[kZUnroll];
#pragma unroll
        for (int u = 0; u < kZUnroll; ++u) {
            const int q = qb + u * kThreads;
            if (q < mine) {
                zv[u] = zsrc[sbase + q];
                rv[u] = d.r[sbase + q];
                if (drift && (q & 7) == 0) prefetch_l2(d.z0 + sbase + q);
                if (Check && (q & 7) == 0) prefetch_l2(d.dxs + sbase + q);
            }
        }
#pragma unroll
        for (int u = 0; u < kZUnroll; ++u) {
            const int q = qb + u * kThreads;
            if (q < mine) vz[q] = zv[u] + rv[u];
        }
    }
    __syncthreads();

    // phase B: the z threshold over the whole block, across the cluster.
    // Each CTA's (sum, count) over its slice goes to part[parity]; after one
    // cluster barrier every CTA adds all ranks' partials in rank order, so
    // every CTA takes the same decisions.  The two parities let a round write
    // its partials while no CTA can still be reading that buffer.
    int parity = 0;
    auto active = [&](double th, double& S, int& C) {
        double b[2] = {0.0, 0.0};
        for (int q = threadIdx.x; q < mine; q += kThreads) {
            const double x = double(vval(q));
            if (th == -INFINITY || x > th) {
                b[0] += x;
                b[1] += 1.0;
            }
        }
        double t[2];
        cluster_sums<2, kThreads / 32>(b, slots, tot, parity, cluster, csize, t);
        S = t[0];
        C = int(t[1]);
        parity ^= 1;
    };
    const double thz = michelot(active, d.n * len, double(d.k0), d.thz[s]);
    cluster.sync();   // no CTA leaves while another may still read its partials
    if (rank == 0 && threadIdx.x == 0) d.thz[s] = thz;

    // phase C: z
    for (int qb = threadIdx.x; qb < mine; qb += kThreads * kZUnroll) {
        Real z1v[kZUnroll], zav[kZUnroll], dxv[kZUnroll];
#pragma unroll
        for (int u = 0; u < kZUnroll; ++u) {
            const int q = qb + u * kThreads;
            if (q < mine) {
                z1v[u] = zsrc[sbase + q];
                zav[u] = drift ? d.z0[sbase + q] : z1v[u];
                if (Check) dxv[u] = d.dxs[sbase + q];
            }
        }
#pragma unroll
        for (int u = 0; u < kZUnroll; ++u) {
            const int q = qb + u * kThreads;
            if (q >= mine) continue;
            const long long e = sbase + q;
            const Real z2 = Real(fmax(double(vval(q)) - thz, 0.0));
            const Real z1 = z1v[u], za = Reflect ? zav[u] : z1;
            d.zh[e] = vanilla ? z2 : lwn * (Real(2) * z2 - z1) + rwn * za;
            if (!Reflect && !vanilla) d.z0[e] = z1;
            if (Check) {
                if (Reflect) d.z2s[e] = z2;
                const double dz = double(z1) - double(z2), dr = double(z1) - double(zav[u]);
                acc[0] += dz * dz;
                acc[1] += double(dxv[u]) * dz;
                acc[2] += dr * dr;
            }
        }
    }
    if (Check) {
        block_sums<3>(acc, scratch, acc);
        if (threadIdx.x == 0) {
            for (int k = 0; k < 3; ++k) d.pyz[(size_t(s) * csize + rank) * 3 + k] = acc[k];
        }
    }
}

// z half-step (solver.py:423) for the pair of period blocks s = pair and
// s = Tp - 1 - pair (N (Tp - s) entries each, N (Tp + 1) together, so every
// pair is the same work), one cluster of `csize` CTAs per pair; CTA `rank`
// owns rows [r0, r1) of both blocks, a contiguous slice of each.  z + r of
// the slices goes to shared memory; each block's threshold comes from its own
// Michelot rounds, the two blocks' rounds taken together, so one cluster
// barrier passes both blocks' (sum, count) through distributed shared memory;
// then the slices' z is written.  Every per-block sum is taken in z_task's
// order, so the results are z_task's, bit for bit; the check partials go to
// each block's own rows of pyz.  Half the clusters of z_task, each with twice
// the entries per barrier: it pays when the pairs still fill the GPU and
// the CTAs are few per SM (FP64, register-bound to one per SM).
template <class Real, int kThreads, bool Reflect, bool Check>
__device__ __forceinline__ void z_task_pair(const Dev<Real>& d, int pair, const Real* zsrc, int step, int gate) {
    const Control* c = d.ctl;
    if (skip(c, gate)) return;   // uniform over the cluster: c is not written here
    ZGroup<false> cluster;
    const int csize = d.csize;
    const int rank = cluster.rank();
    const int r0 = int((long long)d.n * rank / csize), r1 = int((long long)d.n * (rank + 1) / csize);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real* vz = reinterpret_cast<Real*>(smem_raw);
    __shared__ double slots[2][kThreads / 32][4];
    __shared__ double tots[2 * 4];
    __shared__ double scratch[6 * 32];
    const double kn = Reflect ? double(c->restart_iter + step + 2) : 1.0;
    const Real lwn = Real(kn / (kn + 1.0)), rwn = Real(1.0 / (kn + 1.0));
    const bool vanilla = !Reflect && (gate & kGateVanilla);   // as in the y half-step
    const bool drift = Reflect || (gate & kGateDrift);
    const int sblk[2] = {pair, d.tp - 1 - pair};
    int len[2], mine[2], off[2];
    long long sbase[2];
#pragma unroll
    for (int g = 0; g < 2; ++g) {
        len[g] = d.tp - sblk[g];
        mine[g] = (r1 - r0) * len[g];
        sbase[g] = blk(d.n, d.tp, sblk[g]) + (long long)r0 * len[g];
    }
    off[0] = 0;
    off[1] = mine[0];
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};   // per block: |dz|^2, <dx, dz>, drift

    const bool staged = d.zstaged != 0;
    // v(g, q) = z + r of element q of block g's slice, in the same arithmetic either way
    auto vval = [&](int g, int q) -> Real {
        return staged ? vz[off[g] + q] : Real(zsrc[sbase[g] + q] + d.r[sbase[g] + q]);
    };

    // phase A: z + r of the slices into shared memory, kZUnroll loads in flight
#pragma unroll
    for (int g = 0; g < 2; ++g) {
        for (int qb = threadIdx.x; staged && qb < mine[g]; qb += kThreads * kZUnroll) {
            Real zv[kZUnroll], rv[kZUnroll];
#pragma unroll
            for (int u = 0; u < kZUnroll; ++u) {
                const int q = qb + u * kThreads;
                if (q < mine[g]) {
                    zv[u] = zsrc[sbase[g] + q];
                    rv[u] = d.r[sbase[g] + q];
                    if (drift && (q & 7) == 0) prefetch_l2(d.z0 + sbase[g] + q);
                    if (Check && (q & 7) == 0) prefetch_l2(d.dxs + sbase[g] + q);
                }
            }
#pragma unroll
            for (int u = 0; u < kZUnroll; ++u) {
                const int q = qb + u * kThreads;
                if (q < mine[g]) vz[off[g] + q] = zv[u] + rv[u];
            }
        }
    }
    __syncthreads();

    // phase B: each block's z threshold across the cluster.  Each CTA's
    // (sum, count) per block over its slice goes to part[parity]; after one
    // cluster barrier every CTA adds all ranks' partials in rank order, so
    // every CTA takes the same decisions.  The two parities let a round write
    // its partials while no CTA can still be reading that buffer.
    MichelotSteps ms[2];
#pragma unroll
    for (int g = 0; g < 2; ++g) ms[g].init(double(d.k0), d.thz[sblk[g]], d.n * len[g]);
    int parity = 0;
    while (!ms[0].done() || !ms[1].done()) {
        double b[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int g = 0; g < 2; ++g) {
            if (ms[g].done()) continue;
            const double th = ms[g].th;
            for (int q = threadIdx.x; q < mine[g]; q += kThreads) {
                const double x = double(vval(g, q));
                if (th == -INFINITY || x > th) {
                    b[2 * g] += x;
                    b[2 * g + 1] += 1.0;
                }
            }
        }
        double tot[4];
        cluster_sums<4, kThreads / 32>(b, slots, tots, parity, cluster, csize, tot);
#pragma unroll
        for (int g = 0; g < 2; ++g)
            if (!ms[g].done()) ms[g].feed(tot[2 * g], int(tot[2 * g + 1]));
        parity ^= 1;
    }
    cluster.sync();   // no CTA leaves while another may still read its partials
    if (rank == 0 && threadIdx.x == 0) {
        d.thz[sblk[0]] = ms[0].th;
        d.thz[sblk[1]] = ms[1].th;
    }

    // phase C: z
#pragma unroll
    for (int g = 0; g < 2; ++g) {
        const double thz = ms[g].th;
        for (int qb = threadIdx.x; qb < mine[g]; qb += kThreads * kZUnroll) {
            Real z1v[kZUnroll], zav[kZUnroll], dxv[kZUnroll];
#pragma unroll
            for (int u = 0; u < kZUnroll; ++u) {
                const int q = qb + u * kThreads;
                if (q < mine[g]) {
                    z1v[u] = zsrc[sbase[g] + q];
                    zav[u] = drift ? d.z0[sbase[g] + q] : z1v[u];
                    if (Check) dxv[u] = d.dxs[sbase[g] + q];
                }
            }
#pragma unroll
            for (int u = 0; u < kZUnroll; ++u) {
                const int q = qb + u * kThreads;
                if (q >= mine[g]) continue;
                const long long e = sbase[g] + q;
                const Real z2 = Real(fmax(double(vval(g, q)) - thz, 0.0));
                const Real z1 = z1v[u], za = Reflect ? zav[u] : z1;
                d.zh[e] = vanilla ? z2 : lwn * (Real(2) * z2 - z1) + rwn * za;
                if (!Reflect && !vanilla) d.z0[e] = z1;
                if (Check) {
                    if (Reflect) d.z2s[e] = z2;
                    const double dz = double(z1) - double(z2), dr = double(z1) - double(zav[u]);
                    acc[3 * g] += dz * dz;
                    acc[3 * g + 1] += double(dxv[u]) * dz;
                    acc[3 * g + 2] += dr * dr;
                }
            }
        }
    }
    if (Check) {
        block_sums<6>(acc, scratch, acc);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int g = 0; g < 2; ++g)
                for (int k = 0; k < 3; ++k) d.pyz[(size_t(sblk[g]) * csize + rank) * 3 + k] = acc[3 * g + k];
        }
    }
}

template <class Real, int kThreads, bool Reflect, bool Check, bool Pair>
__global__ void __launch_bounds__(kThreads)
z_kernel(Dev<Real> d, const Real* zsrc, int step, int gate) {
    if constexpr (Pair)
        z_task_pair<Real, kThreads, Reflect, Check>(d, int(blockIdx.x) / d.csize, zsrc, step, gate);
    else
        z_task<Real, kThreads, Reflect, Check>(d, int(blockIdx.x) / d.csize, zsrc, step, gate);
}

// The FP32 z kernel with registers capped for three CTAs per SM (two at its
// natural 56): 2-3.5 % faster PRIA solves at T >= 500, neutral below; in FP64
// the cap spills and was 2-4 % slower, so z_kernel<double> keeps its own.
template <int kThreads, bool Reflect, bool Check, bool Pair>
__global__ void __launch_bounds__(kThreads, 1536 / kThreads)
z_kernel_f32(Dev<float> d, const float* zsrc, int step, int gate) {
    if constexpr (Pair)
        z_task_pair<float, kThreads, Reflect, Check>(d, int(blockIdx.x) / d.csize, zsrc, step, gate);
    else
        z_task<float, kThreads, Reflect, Check>(d, int(blockIdx.x) / d.csize, zsrc, step, gate);
}

// the z kernel a precision launches
template <class Real, int kThreads, bool Reflect, bool Check, bool Pair>
constexpr auto z_entry() {
    if constexpr (sizeof(Real) == 4)
        return z_kernel_f32<kThreads, Reflect, Check, Pair>;
    else
        return z_kernel<Real, kThreads, Reflect, Check, Pair>;
}

// The primal bound terms at x for period block s (solver.py:347-365):
// sum_i K_i max_{t>=s} x_ist, K0 max_{i, t>=s} x_ist and sum h x over the
// block, restricted to t < tlimit and s < tlimit (tlimit = t for the unpadded
// objective).  `force` runs it after termination.
template <class Real>
__device__ __forceinline__ void upper_kernel_tile(const Dev<Real>& d, int tile, const Real* x, int tlimit, int force) {
    if (!force && d.ctl->terminated) return;
    __shared__ double scratch[3 * 32];
    __shared__ double wmax[32];
    const int s = tile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    double acc[3] = {0.0, 0.0, 0.0};
    double bmax = 0.0;
    if (s < tlimit && index_ok(blk(d.n, d.tp, s) + (long long)d.n * (d.tp - s) <= d.nd, &d.ctl->status)) {
        const int len = d.tp - s, valid = tlimit - s;
        const long long base = blk(d.n, d.tp, s);
        for (int i = warp; i < d.n; i += nwarps) {
            const long long e0 = base + (long long)i * len;
            double mx = 0.0, hx = 0.0;
            // chunks of 8 predicated loads per lane: one round trip each
            for (int q0 = 0; q0 < valid; q0 += 32 * 8) {   // uniform over the warp
                Real xv[8], hv[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int q = q0 + lane + 32 * u;
                    if (q < valid) {
                        xv[u] = x[e0 + q];
                        hv[u] = d.h[e0 + q];
                    }
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    if (q0 + lane + 32 * u >= valid) continue;
                    const double v = double(xv[u]);
                    mx = fmax(mx, v);
                    hx += double(hv[u]) * v;
                }
            }
            mx = warp_max(mx);
            hx = warp_sum(hx);
            if (lane == 0) {
                acc[0] += double(d.k[i]) * mx;
                acc[2] += hx;
                bmax = fmax(bmax, mx);
            }
        }
    }
    if (lane == 0) wmax[warp] = bmax;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < nwarps; ++w) b = fmax(b, wmax[w]);
        acc[1] = double(d.k0) * b;
    }
    block_sums<3>(acc, scratch, acc);
    if (threadIdx.x == 0) {
        for (int k = 0; k < 3; ++k) d.pup[size_t(s) * 3 + k] = acc[k];
    }
}

template <class Real>
__global__ void __launch_bounds__(kAuxThreads)
upper_kernel(Dev<Real> d, const Real* __restrict__ x, int tlimit, int force) {
    upper_kernel_tile<Real>(d, blockIdx.x, x, tlimit, force);
}

// The dual bound sum_{i,t} min_{s<=t} (h + y + z) (solver.py:388-402) for one
// tile of kLowTW columns of one item.
template <class Real>
__device__ __forceinline__ void lower_kernel_tile(const Dev<Real>& d, int tile, const Real* y, const Real* z) {
    if (d.ctl->terminated) return;
    __shared__ double cmin[kAuxThreads / 32][kLowTW];
    __shared__ double scratch[32];
    const int item = tile % d.n;
    const int ctile = d.ntc_low - 1 - int(tile / d.n);
    const int t0 = ctile * kLowTW;
    const int tcols = min(kLowTW, d.tp - t0);
    const int rows = t0 + tcols;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int tt = t0 + lane;
    double mn = INFINITY;
    // four rows per warp in flight (a minimum: the order does not matter)
    for (int s0 = warp; s0 < rows; s0 += 4 * nwarps) {
        Real hv[4], yv[4], zv[4];
        bool in[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int s = s0 + u * nwarps;
            in[u] = s < rows && lane < tcols && tt >= s &&
                    index_ok(blk(d.n, d.tp, s) + (long long)item * (d.tp - s) + (tt - s) < d.nd, &d.ctl->status);
            if (in[u]) {
                const long long e = blk(d.n, d.tp, s) + (long long)item * (d.tp - s) + (tt - s);
                hv[u] = d.h[e];
                yv[u] = y[e];
                zv[u] = z[e];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (in[u]) mn = fmin(mn, (double(hv[u]) + double(yv[u])) + double(zv[u]));
    }
    cmin[warp][lane] = mn;
    __syncthreads();
    double acc[1] = {0.0};
    if (warp == 0 && lane < tcols) {
        double v = INFINITY;
        for (int w = 0; w < nwarps; ++w) v = fmin(v, cmin[w][lane]);
        acc[0] = v;
    }
    block_sums<1>(acc, scratch, acc);
    if (threadIdx.x == 0) d.plo[tile] = acc[0];
}

template <class Real>
__global__ void __launch_bounds__(kAuxThreads)
lower_kernel(Dev<Real> d, const Real* __restrict__ y, const Real* __restrict__ z) {
    lower_kernel_tile<Real>(d, blockIdx.x, y, z);
}

__device__ __forceinline__ double canonical(const double* xs, const double* yzs, double omega,
                                            double eta) {
    const double v = (omega / eta) * xs[0] + (1.0 / (eta * omega)) * yzs[0] - 2.0 * yzs[1];
    return sqrt(v > 0.0 ? v : 0.0);
}

__device__ __forceinline__ bool should_stop(double gap, long long iteration, const Params& p) {
    const bool within = iteration < p.max_iter || p.max_iter < 0;
    return !(within && !(gap <= p.tolerance));   // NaN keeps going
}

// mode 0: the check before the loop; 1: after an op_steps block; 2: after the
// restart step (solver.py:514-594); 3: after a block of vanilla steps (the
// bounds at the current point, solver.py:601-606); 4: after the step that
// ends the vanilla phase and starts the Halpern one (the primal weight from
// the drift of the vanilla phase, solver.py:680-694).
__device__ __forceinline__ void check_body(Control* c, Params p, const double* px, int nbx, const double* py,
                                           int nby, const double* pyz, int nbyz, const double* pup, int nbup,
                                           const double* plo, int nblo, int mode) {
    if (c->terminated) return;
    if (mode == 2 && !c->restart) return;
    __shared__ double scratch[3 * 32];
    __shared__ double xs[2], yzs[3], ys_[3], up[3], lo[1];
    if (mode != 3) {
        reduce_rows<2>(px, nbx, scratch, xs);
        reduce_rows<3>(py, nby, scratch, ys_);
        reduce_rows<3>(pyz, nbyz, scratch, yzs);
        if (threadIdx.x == 0)
            for (int k = 0; k < 3; ++k) yzs[k] += ys_[k];   // y parts + z parts, in that order
    }
    if (mode != 2 && mode != 4) {
        reduce_rows<3>(pup, nbup, scratch, up);
        reduce_rows<1>(plo, nblo, scratch, lo);
    }
    if (threadIdx.x != 0) return;
    if (mode == 4) {
        // omega = |d(y, z)| / |dx| over the vanilla phase, NaN -> the initial one
        if (c->iteration > 0) {
            const double om = sqrt(yzs[2]) / sqrt(xs[1]);
            c->omega = isnan(om) ? p.omega0 : om;
        }
        c->fp_error = canonical(xs, yzs, c->omega, p.eta);
        c->new_error = c->fp_error;
        c->check_error = INFINITY;
        c->restart_iter = 0;
        c->restart = 0;
        c->phase_done = 0;
        c->result_slot = 1;   // the point the gap was measured at is now the anchor
        c->terminated = should_stop(c->gap, c->iteration, p) ? 1 : 0;
        trace_put(p.trace, p.trace_cap, c->trace_len, c->iteration, c->gap, c->fp_error, c->omega, c->lower,
                  c->upper, 5, c->terminated);
        return;
    }
    if (mode == 3) {
        const double upper = (up[0] + up[1] + up[2]) * p.scale;
        const double lower = lo[0] * p.scale;
        const double gap = (upper - lower) / (1.0 + fabs(lower) + fabs(upper));
        c->upper = upper;
        c->lower = lower;
        c->gap = gap;
        c->iteration += p.op_steps;
        c->result_slot = 3;
        const bool within = c->iteration < p.vanilla_max || p.vanilla_max < 0;
        if (!(gap > p.tolerance)) c->terminated = 1;
        else if (!within) {
            if (p.vanilla_solve) c->terminated = 1;   // a vanilla solve: its iteration limit
            else c->phase_done = 1;
        }
        trace_put(p.trace, p.trace_cap, c->trace_len, c->iteration, gap, NAN, c->omega, lower, upper, 4,
                  c->terminated);
        return;
    }
    if (mode == 2) {
        c->fp_error = canonical(xs, yzs, c->omega, p.eta);
        c->check_error = INFINITY;
        c->restart_iter = 0;
        c->restart = 0;
        return;
    }
    const double upper = (up[0] + up[1] + up[2]) * p.scale;
    const double lower = lo[0] * p.scale;
    const double gap = (upper - lower) / (1.0 + fabs(lower) + fabs(upper));
    c->upper = upper;
    c->lower = lower;
    c->gap = gap;
    if (mode == 0) {
        c->fp_error = canonical(xs, yzs, c->omega, p.eta);
        c->new_error = c->fp_error;
        c->check_error = INFINITY;
        Params q = p;
        q.max_iter = p.start_max;
        c->terminated = should_stop(gap, c->iteration, q) ? 1 : 0;
        c->result_slot = 1;
        c->restart = 0;
        trace_put(p.trace, p.trace_cap, c->trace_len, c->iteration, gap, c->fp_error, c->omega, lower, upper, -1,
                  c->terminated);
        return;
    }
    c->iteration += p.op_steps;
    c->restart_iter += p.op_steps;
    const double new_err = canonical(xs, yzs, c->omega, p.eta);
    c->new_error = new_err;
    const bool terminated = should_stop(gap, c->iteration, p);
    const bool sufficient = new_err <= p.beta_sufficient * c->fp_error;
    const bool necessary = new_err <= p.beta_necessary * c->fp_error && new_err > c->check_error;
    const bool artificial = double(c->restart_iter) >= p.beta_artificial * double(c->iteration);
    const bool restart = sufficient || necessary || artificial;
    if (restart) {
        const double pn = sqrt(xs[1]), dn = sqrt(yzs[2]);
        if (pn > 1e-16 && dn > 1e-16) {
            const double th = c->theta;
            c->omega = exp(th * (log(dn) - log(pn)) + (1.0 - th) * log(c->omega));
            c->theta = p.theta_target + p.theta_decay * (th - p.theta_target);
        }
    }
    if (terminated) {
        c->terminated = 1;
        c->result_slot = 2;
        c->restart = 0;
    } else {
        // the gap was measured at the step (x2s, y2s, z2s); a restart step
        // that follows makes that point the anchor and sets result_slot = 1
        c->result_slot = 2;
        if (restart) c->restart = 1;
        else c->check_error = new_err;
    }
    const int kind = (terminated || !restart) ? 0 : (sufficient ? 1 : (necessary ? 2 : 3));
    trace_put(p.trace, p.trace_cap, c->trace_len, c->iteration, gap, new_err, c->omega, lower, upper, kind,
              terminated ? 1 : 0);
}

__global__ void __launch_bounds__(kCheckBlock)
check_kernel(Control* c, Params p, const double* __restrict__ px, int nbx,
             const double* __restrict__ py, int nby,
             const double* __restrict__ pyz, int nbyz, const double* __restrict__ pup, int nbup,
             const double* __restrict__ plo, int nblo, int mode) {
    check_body(c, p, px, nbx, py, nby, pyz, nbyz, pup, nbup, plo, nblo, mode);
}

// ---- the persistent kernel for small instances ----------------------------
// (the reference's megakernel, jrp/pria-cuda/src/solver.cuh:145-312, on this
// file's own half-steps.)  One cooperative launch runs a whole check block:
// op_steps steps of x, then y and z, the bounds, the check and the gated
// restart step, the same tile functions as the per-kernel graph in the same
// order, each phase's units dealt round-robin to the resident CTAs and the
// phases separated by grid barriers (bounded waits, common.cuh).  It replaces
// the graph's 55 kernel boundaries per block by 34 barriers (37 with a
// restart).  A z task is one whole period block in one CTA (ZGroup<true>), so
// instances whose largest block does not fit one CTA's shared memory keep the
// graph.  The tile functions take their iterates through plain pointers (no
// __restrict__): here a buffer one phase reads, another phase of the same
// launch writes, and only the per-kernel wrappers may promise read-only data.
// A barrier that runs out sets Control::status to kMegaWaitStatus.
constexpr int kMegaThreads = 256;   // = kXThreads = kYThreads = kAuxThreads = kCheckBlock
constexpr int kMegaWaitStatus = 1;
#ifndef RB200_PRIA_MEGA_MINB
#define RB200_PRIA_MEGA_MINB 1          // CTAs per SM the kernel is compiled for (sweeps build with -D)
#endif

struct MegaArgs {
    GridBar* bar;
    unsigned expect;                 // CTAs each barrier waits for (the grid)
    unsigned long long wait_ns;      // a barrier's wait limit
};

template <class Real, bool Reflect, bool Check>
__device__ __forceinline__ void mega_x(const Dev<Real>& d, const Real* xs, const Real* ys, const Real* zs, int step,
                                       int gate) {
    const int tiles = d.n * d.ntc;
    for (int tile = int(blockIdx.x); tile < tiles; tile += gridDim.x) {
        x_kernel_tile<Real, kXTile, Reflect, Check>(d, tile, xs, ys, zs, step, gate);
        __syncthreads();   // the next tile reuses the shared tile
    }
}

// Out of line: inlined into the step loop, the z task's register demand grows
// past the budget of the whole kernel.
template <class Real, bool Reflect, bool Check>
__device__ __noinline__ void mega_z(const Dev<Real>& d, int s, const Real* zs, int step, int gate) {
    z_task<Real, kMegaThreads, Reflect, Check, true>(d, s, zs, step, gate);
}

// The z tasks (heaviest first) and then the y tiles of one half-step.
template <class Real, bool Reflect, bool Check>
__device__ __forceinline__ void mega_yz(const Dev<Real>& d, const Real* ys, const Real* zs, int step, int gate) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nby = int(((long long)d.tp * d.n + kYThreads / 32 - 1) / (kYThreads / 32));
    const int units = d.tp + nby;
    for (int u = int(blockIdx.x); u < units; u += gridDim.x) {
        if (u < d.tp)
            mega_z<Real, Reflect, Check>(d, u, zs, step, gate);
        else
            y_kernel_tile<Real, Reflect, Check>(d, u - d.tp, ys, step, gate, reinterpret_cast<Real*>(smem_raw), d.tp);
        __syncthreads();
    }
}

template <class Real>
__device__ __forceinline__ void mega_bounds(const Dev<Real>& d, const Real* x, const Real* y, const Real* z) {
    const int units = d.tp + d.n * d.ntc_low;
    for (int u = int(blockIdx.x); u < units; u += gridDim.x) {
        if (u < d.tp)
            upper_kernel_tile<Real>(d, u, x, d.tp, 0);
        else
            lower_kernel_tile<Real>(d, u - d.tp, y, z);
        __syncthreads();
    }
}

__device__ __forceinline__ void mega_check(Control* c, const Params& prm, const double* px, int nbx, const double* py,
                                           int nby, const double* pyz, int nbyz, const double* pup, int nbup,
                                           const double* plo, int nblo, int mode) {
    if (blockIdx.x == 0) check_body(c, prm, px, nbx, py, nby, pyz, nbyz, pup, nbup, plo, nblo, mode);
}

// The head of a captured check block: the block's body runs only while the
// solve has not terminated (a block queued behind the one that ended the
// solve then costs this one launch instead of its gated kernels).
__global__ void block_gate_kernel(const Control* c, cudaGraphConditionalHandle body) {
    if (threadIdx.x == 0) cudaGraphSetConditional(body, c->terminated ? 0u : 1u);
}

// Vanilla: one block of the vanilla phase (enqueue_vanilla_block's steps);
// otherwise one Halpern check block (enqueue_block's).
template <class Real, bool Vanilla>
__global__ void __launch_bounds__(kMegaThreads, RB200_PRIA_MEGA_MINB)
mega_block_kernel(const __grid_constant__ Dev<Real> d, const __grid_constant__ Params prm, MegaArgs a) {
    const int op = int(prm.op_steps);
    const int nbx = d.n * d.ntc, nblo = d.n * d.ntc_low;
    const int nby = int(((long long)d.tp * d.n + kYThreads / 32 - 1) / (kYThreads / 32));
    auto sync = [&]() {
        if (grid_sync(a.bar, a.expect, a.wait_ns)) return true;
        if (threadIdx.x == 0) d.ctl->status = kMegaWaitStatus;
        return false;
    };
    if constexpr (Vanilla) {
        for (int s = 0; s < op; ++s) {
            mega_x<Real, false, false>(d, d.xh, d.yh, d.zh, 0, kGateVanilla);
            if (!sync()) return;
            mega_yz<Real, false, false>(d, d.yh, d.zh, 0, kGateVanilla);
            if (!sync()) return;
        }
        mega_bounds<Real>(d, d.xh, d.yh, d.zh);
        if (!sync()) return;
        mega_check(d.ctl, prm, d.px, nbx, d.py, nby, d.pyz, d.tp, d.pup, d.tp, d.plo, nblo, 3);
    } else {
        for (int s = 0; s < op; ++s) {
            if (s + 1 < op)
                mega_x<Real, true, false>(d, d.xh, d.yh, d.zh, s, 0);
            else
                mega_x<Real, true, true>(d, d.xh, d.yh, d.zh, s, 0);
            if (!sync()) return;
            if (s + 1 < op)
                mega_yz<Real, true, false>(d, d.yh, d.zh, s, 0);
            else
                mega_yz<Real, true, true>(d, d.yh, d.zh, s, 0);
            if (!sync()) return;
        }
        mega_bounds<Real>(d, d.x2s, d.y2s, d.z2s);
        if (!sync()) return;
        mega_check(d.ctl, prm, d.px, nbx, d.py, nby, d.pyz, d.tp, d.pup, d.tp, d.plo, nblo, 1);
        if (!sync()) return;
        if (!d.ctl->restart) return;   // uniform: the check above is the last writer
        mega_x<Real, false, true>(d, d.x2s, d.y2s, d.z2s, 0, kGateRestart);
        if (!sync()) return;
        mega_yz<Real, false, true>(d, d.y2s, d.z2s, 0, kGateRestart);
        if (!sync()) return;
        mega_check(d.ctl, prm, d.px, nbx, d.py, nby, d.pyz, d.tp, d.pup, d.tp, d.plo, nblo, 2);
    }
}

// The start point: the projection of zero, i.e. each simplex's centre:
// x = 1/(t+1), y = K_i/(Tp-s), z = K0/(N(Tp-s)) (solver.py:669-671), one CTA
// per period block.  Also resets the control block.
template <class Real>
__global__ void init_kernel(Dev<Real> d, Control* c, double omega, double theta) {
    const int s = blockIdx.x;
    const int len = d.tp - s;
    const long long base = blk(d.n, d.tp, s);
    const long long count = (long long)d.n * len;
    const Real zc = d.k0 > Real(0) ? Real(double(d.k0) / double(count)) : Real(0);
    for (long long q = threadIdx.x; q < count; q += blockDim.x) {
        const int i = int(q / len), t = s + int(q % len);
        const Real kv = d.k[i];
        d.x0[base + q] = Real(1.0 / double(t + 1));
        d.y0[base + q] = kv > Real(0) ? Real(double(kv) / double(len)) : Real(0);
        d.z0[base + q] = zc;
    }
    if (s == 0 && threadIdx.x == 0) {
        c->omega = omega;
        c->theta = theta;
        c->fp_error = 0.0;
        c->check_error = INFINITY;
        c->new_error = 0.0;
        c->lower = c->upper = c->gap = NAN;
        c->restart_iter = 0;
        c->iteration = 0;
        c->terminated = 0;
        c->restart = 0;
        c->result_slot = 1;
        c->status = 0;
        c->phase_done = 0;
        c->trace_len = 0;
    }
}

// Warm start: dense [n][t][t] (normalised duals) -> the packed layout, duals
// scaled back onto the K_i / K0 simplices (solver.py:662-671); zero padding.
template <class Real>
__global__ void warm_pack_kernel(Dev<Real> d, const double* __restrict__ wx, const double* __restrict__ wy,
                                 const double* __restrict__ wz, Real* __restrict__ px, Real* __restrict__ py,
                                 Real* __restrict__ pz) {
    const int s = blockIdx.x;
    const int len = d.tp - s;
    const long long base = blk(d.n, d.tp, s);
    const long long count = (long long)d.n * len;
    for (long long q = threadIdx.x; q < count; q += blockDim.x) {
        const int i = int(q / len), t = s + int(q % len);
        Real vx = Real(0), vy = Real(0), vz = Real(0);
        if (s < d.t && t < d.t) {
            const long long g = ((long long)i * d.t + s) * d.t + t;
            vx = Real(wx[g]);
            vy = Real(wy[g] * double(d.k[i]));
            vz = Real(wz[g] * double(d.k0));
        }
        px[base + q] = vx;
        py[base + q] = vy;
        pz[base + q] = vz;
    }
}

// Projections of a packed point onto X, Y, Z (for a warm start): the column,
// row and block passes of the step kernels with nothing else around them.
template <class Real, int TW>
__global__ void __launch_bounds__(kXThreads) project_x_kernel(Dev<Real> d, Real* x) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* pre = reinterpret_cast<double*>(smem_raw);
    __shared__ double theta[TW];
    const int item = blockIdx.x % d.n;
    const int ctile = d.ntc - 1 - int(blockIdx.x / d.n);
    const int t0 = ctile * TW;
    const int tcols = min(TW, d.tp - t0);
    const int rows = t0 + tcols;
    const int stride = rows | 1;
    constexpr int kRpw = 32 / TW;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int col = lane % TW, sub = lane / TW;
    const int tt = t0 + col;
    for (int s = warp * kRpw + sub; s < rows; s += nwarps * kRpw)
        if (col < tcols && tt >= s) pre[col * stride + s] = x[blk(d.n, d.tp, s) + (long long)item * (d.tp - s) + (tt - s)];
    __syncthreads();
    for (int cc = warp; cc < tcols; cc += nwarps) {
        const double th = michelot_smem(pre + cc * stride, t0 + cc + 1, 1.0, NAN);
        if (lane == 0) theta[cc] = th;
    }
    __syncthreads();
    for (int s = warp * kRpw + sub; s < rows; s += nwarps * kRpw)
        if (col < tcols && tt >= s)
            x[blk(d.n, d.tp, s) + (long long)item * (d.tp - s) + (tt - s)] =
                Real(fmax(pre[col * stride + s] - theta[col], 0.0));
}

template <class Real>
__global__ void __launch_bounds__(kAuxThreads) project_yz_kernel(Dev<Real> d, Real* y, Real* z) {
    // one CTA per block s: y rows by warps, then z over the whole block
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double scratch[2 * 32];
    const int s = blockIdx.x;
    const int len = d.tp - s;
    const long long base = blk(d.n, d.tp, s);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int i = warp; i < d.n; i += nwarps) {
        const long long e0 = base + (long long)i * len;
        Real v[32];
#pragma unroll
        for (int k = 0; k < 32; ++k)
            if (lane + 32 * k < len) v[k] = y[e0 + lane + 32 * k];
        const double th = michelot_regs(v, len, double(d.k[i]), NAN);
#pragma unroll
        for (int k = 0; k < 32; ++k)
            if (lane + 32 * k < len) y[e0 + lane + 32 * k] = Real(fmax(double(v[k]) - th, 0.0));
    }
    // z: the whole block through global memory (a one-off projection)
    const long long count = (long long)d.n * len;
    const double target = double(d.k0);
    double th = INFINITY;
    if (target > 0.0) {
        double a[2] = {0.0, 0.0};
        for (long long q = threadIdx.x; q < count; q += blockDim.x) a[0] += double(z[base + q]);
        block_sums<2>(a, scratch, a);
        __shared__ double bc[2];
        if (threadIdx.x == 0) bc[0] = a[0];
        __syncthreads();
        th = (bc[0] - target) / double(count);
        double cnt = double(count);
        for (long long round = 0; round < count; ++round) {
            double b[2] = {0.0, 0.0};
            for (long long q = threadIdx.x; q < count; q += blockDim.x) {
                const double x = double(z[base + q]);
                if (x > th) {
                    b[0] += x;
                    b[1] += 1.0;
                }
            }
            block_sums<2>(b, scratch, b);
            if (threadIdx.x == 0) {
                bc[0] = b[0];
                bc[1] = b[1];
            }
            __syncthreads();
            const double S2 = bc[0], C2 = bc[1];
            __syncthreads();
            if (C2 >= cnt || C2 == 0.0) break;
            cnt = C2;
            th = (S2 - target) / C2;
        }
    }
    for (long long q = threadIdx.x; q < count; q += blockDim.x)
        z[base + q] = Real(fmax(double(z[base + q]) - th, 0.0));
    (void)smem_raw;
}

// Packed -> dense [n][t][t] output, unpadded; y / K_i and z / K0 (zero when
// the budget is zero), mode 0 x, 1 y, 2 z.
template <class Real, class Out>
__global__ void unpack_kernel(Dev<Real> d, const Real* __restrict__ src, int mode, Out* __restrict__ out) {
    const long long total = (long long)d.n * d.t * d.t;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
        const int t = int(g % d.t);
        const int s = int((g / d.t) % d.t);
        const int i = int(g / ((long long)d.t * d.t));
        double v = 0.0;
        if (t >= s) {
            v = double(src[blk(d.n, d.tp, s) + (long long)i * (d.tp - s) + (t - s)]);
            if (mode == 1) v = d.k[i] > Real(0) ? v / double(d.k[i]) : 0.0;
            if (mode == 2) v = d.k0 > Real(0) ? v / double(d.k0) : 0.0;
        }
        out[g] = Out(v);
    }
}

// Input: dense H -> sum of squares of its upper triangle (fixed grid, fixed
// order) and the packed, scaled h.
template <class In>
__global__ void h_squares_kernel(int n, int t, const In* __restrict__ H, double* __restrict__ partial) {
    __shared__ double scratch[32];
    const long long total = (long long)n * t * t;
    const long long stride = (long long)gridDim.x * blockDim.x;
    double acc[1] = {0.0};
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
        const int tt = int(g % t), s = int((g / t) % t);
        if (tt >= s) {
            const double v = double(H[g]);
            acc[0] += v * v;
        }
    }
    block_sums<1>(acc, scratch, acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
}

template <class In, class Real>
__global__ void h_pack_kernel(Dev<Real> d, const In* __restrict__ H, double inv_scale, Real* __restrict__ h) {
    const int s = blockIdx.x;
    const int len = d.tp - s;
    const long long base = blk(d.n, d.tp, s);
    const long long count = (long long)d.n * len;
    for (long long q = threadIdx.x; q < count; q += blockDim.x) {
        const int i = int(q / len), t = s + int(q % len);
        double v = 0.0;
        if (s < d.t && t < d.t) v = double(H[((long long)i * d.t + s) * d.t + t]) * inv_scale;
        h[base + q] = Real(v);
    }
}

// Demand-form holding costs: h[i, s, t] = rate_i d_it (t - s) / scale for
// s <= t < T, zero on the pad period.
template <class Real>
__global__ void h_demand_kernel(Dev<Real> d, const double* __restrict__ rate, const double* __restrict__ demand,
                                double inv_scale, Real* __restrict__ h) {
    const int s = blockIdx.x;
    const int len = d.tp - s;
    const long long base = blk(d.n, d.tp, s);
    const long long count = (long long)d.n * len;
    for (long long q = threadIdx.x; q < count; q += blockDim.x) {
        const int i = int(q / len), t = s + int(q % len);
        double v = 0.0;
        if (s < d.t && t < d.t) v = rate[i] * demand[(long long)i * d.t + t] * double(t - s) * inv_scale;
        h[base + q] = Real(v);
    }
}

constexpr int kSquareBlocks = 296;

__global__ void sum_rows_kernel(const double* __restrict__ partial, int count, double* out) {
    __shared__ double scratch[32];
    __shared__ double total[1];
    reduce_rows<1>(partial, count, scratch, total);
    if (threadIdx.x == 0) *out = total[0];
}

// ---------------------------------------------------------------------------
// host side

// reform_pria_run's return value when the wall-clock budget ran out.
constexpr int kStatusTimeLimit = REFORM_PRIA_STATUS_TIME_LIMIT;
constexpr int kStatusBounds = REFORM_PRIA_STATUS_BOUNDS;

struct SolverBase {
    // Wall-clock budget of each run, in seconds; < 0: none.  Checked on the
    // host each time a check's result arrives.
    double time_limit = -1.0;
    virtual ~SolverBase() = default;
    virtual int run() = 0;
    virtual int result(double* x, double* y, double* z, pria_result_info* info) = 0;
    virtual int result_f32(float* x, float* y, float* z, pria_result_info* info) = 0;
    virtual int set_warm(const double* wx, const double* wy, const double* wz) = 0;
    virtual long long launches() const = 0;
    virtual int run_profiled(double* ms, long long* count) = 0;
    // -1 auto, 0 the graph, 1 the persistent kernel where the instance allows
    // it; *active: which one later runs take
    virtual int set_megakernel(int mode, int* active) = 0;
    virtual int set_trace(int capacity) = 0;
    virtual int get_trace(reform_trace_record* out, int capacity, int64_t* total) = 0;
};

template <class Real>
struct Solver final : SolverBase {
    int n = 0, t = 0, tp = 0;
    long long nd = 0;
    pria_params p{};
    Params prm{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int stream_dev = -1;   // the device of an owned stream (from the library's stream pool)
    PoolBuf<Real> h, k, xh, x0, r, yh, y0, zh, z0, x2s, dxs, y2s, z2s;
    PoolBuf<double> px, py, pyz, pup, plo, final_up, thx, thy, thz;
    PoolBuf<double> warm[3];   // dense warm start (FP64), optional
    bool has_warm = false;
    PoolBuf<Control> ctl;
    Control* mirror = nullptr;
    Dev<Real> d{};
    int tw = kXTile, nbx = 1, nby = 1, nbyz = 1, nblo = 1;
    size_t x_smem = 0, yz_smem = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t done[2] = {nullptr, nullptr};
    long long nlaunch = 0, block_nodes = 0;
    bool gated = false;   // the captured block is the conditional (gated) graph
    int runs = 0;
    // The persistent kernel (mega_block_kernel) in place of the graph: chosen
    // at set-up (mode -1: at most kMegaAutoEntries packed entries), or forced
    // by set_mega; mega_grid resident CTAs of mega_smem bytes each.
    bool mega = false;
    int mega_mode = -1;              // -1 auto, 0 off, 1 on where the instance allows it
    int mega_grid = 0;
    size_t mega_smem = 0;
    unsigned mega_phantom = 0;       // CTAs the barriers also wait for, never launched (fault injection)
    unsigned long long mega_wait_ns = 1000000000ull;
    PoolBuf<GridBar> bar;
    PoolBuf<reform_trace_record> trace;   // the convergence-trace ring, optional
    static constexpr size_t kMegaSmemLimit = 96 * 1024;
    static constexpr long long kMegaAutoEntries = 16384;
    static constexpr int kZThreadsPerCta = z_threads<Real>();
    // y rows: one padded row of at most kMaxPeriods reals per warp
    static constexpr size_t y_smem_limit() { return size_t(kYThreads / 32) * kMaxPeriods * sizeof(Real); }
    // x tiles: kXTile columns of a padded row of at most kMaxPeriods (+1)
    // FP64 values
    // z tasks of the z half-step (pairs of period blocks, or blocks)
    int z_tasks() const { return d.zpair ? tp / 2 : tp; }
    static constexpr size_t x_smem_limit() {
        return size_t(kXTile) * size_t(kMaxPeriods + 1) * sizeof(double);
    }

    ~Solver() override {
        if (stream) cudaStreamSynchronize(stream);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto& ev : done) if (ev) cudaEventDestroy(ev);
        for (auto& ev : evpool) cudaEventDestroy(ev);
        for (auto* b : {&h, &k, &xh, &x0, &r, &yh, &y0, &zh, &z0, &x2s, &dxs, &y2s, &z2s}) b->release();
        for (auto* b : {&px, &py, &pyz, &pup, &plo, &final_up, &thx, &thy, &thz}) b->release();
        for (auto& b : warm) b.release();
        bar.release();
        trace.release();
        ctl.release();
        if (stream) cudaStreamSynchronize(stream);
        pinned_put(mirror);
        if (own_stream && stream) stream_put(stream, stream_dev);
    }

    cudaError_t begin(int64_t n_, int64_t t_, cudaStream_t s) {
        (void)cudaGetLastError();   // a stale error of an unrelated earlier call is not ours
        n = int(n_);
        t = int(t_);
        tp = t + (t & 1);
        nd = (long long)n * tp * (tp + 1) / 2;
        if (s) {
            stream = s;
        } else {
            RB_CUDA_TRY(stream_get(&stream, &stream_dev));
            own_stream = true;
        }
        mirror = static_cast<Control*>(pinned_get());
        if (!mirror) return cudaErrorMemoryAllocation;
        std::memset(static_cast<void*>(mirror), 0, sizeof(Control));   // no run yet: no trace, nothing done
        return cudaSuccess;
    }

    // The scaled K on the device and the scalar fields of the descriptor.
    template <class In>
    cudaError_t set_costs(const In* K, double K0, double hsq) {
        double ss = K0 * K0 + hsq;
        for (int i = 0; i < n; ++i) ss += double(K[i]) * double(K[i]);
        prm.scale = ss > 0.0 ? std::sqrt(ss) : 1.0;
        std::vector<Real> ks(n);
        for (int i = 0; i < n; ++i) ks[i] = Real(double(K[i]) / prm.scale);
        RB_CUDA_TRY(k.upload(ks.data(), n, stream));
        RB_CUDA_TRY(h.alloc(nd, stream));
        d.n = n; d.t = t; d.tp = tp; d.nd = nd;
        d.k = k.ptr;
        d.k0 = Real(K0 / prm.scale);
        return cudaSuccess;
    }

    // Demand-form holding costs H_ist = rate_i d_it (t - s): the packed h is
    // built on the device from N + N T numbers, and sum H^2 on the host as
    // sum_i rate_i^2 sum_t d_it^2 sum_{s<=t} (t - s)^2.
    cudaError_t setup_demand(int64_t n_, int64_t t_, const double* K, double K0, const double* rate,
                             const double* demand, cudaStream_t s) {
        RB_CUDA_TRY(begin(n_, t_, s));
        double hsq = 0.0;
        for (int i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int tt = 0; tt < t; ++tt) {
                const double dd = demand[(long long)i * t + tt], lag = double(tt);
                acc += dd * dd * (lag * (lag + 1.0) * (2.0 * lag + 1.0) / 6.0);
            }
            hsq += rate[i] * rate[i] * acc;
        }
        RB_CUDA_TRY(set_costs<double>(K, K0, hsq));
        {
            PoolBuf<double> rd, dd;
            RB_CUDA_TRY(rd.upload(rate, n, stream));
            RB_CUDA_TRY(dd.upload(demand, size_t(n) * t, stream));
            h_demand_kernel<Real><<<tp, 256, 0, stream>>>(d, rd.ptr, dd.ptr, 1.0 / prm.scale, h.ptr);
            RB_CUDA_TRY(cudaGetLastError());
        }
        return setup_common();
    }

    template <class In>
    cudaError_t setup(int64_t n_, int64_t t_, const In* K, double K0, const In* H, cudaStream_t s) {
        RB_CUDA_TRY(begin(n_, t_, s));
        // scale = ||(triu H, K, K0)||_2 (solver.py:652-654)
        double hsq = 0.0;
        {
            PoolBuf<In> Hd;
            PoolBuf<double> part, tot;
            // H (n t^2 values, the bulk of a solve's input) through the pinned
            // staging ring
            RB_CUDA_TRY(Hd.alloc(size_t(n) * t * t, stream));
            RB_CUDA_TRY(staged_upload(Hd.ptr, H, sizeof(In) * size_t(n) * t * t, stream));
            RB_CUDA_TRY(part.alloc(kSquareBlocks, stream));
            RB_CUDA_TRY(tot.alloc(1, stream));
            h_squares_kernel<In><<<kSquareBlocks, 256, 0, stream>>>(n, t, Hd.ptr, part.ptr);
            sum_rows_kernel<<<1, 256, 0, stream>>>(part.ptr, kSquareBlocks, tot.ptr);
            double* hp = reinterpret_cast<double*>(mirror);
            RB_CUDA_TRY(cudaMemcpyAsync(hp, tot.ptr, sizeof(double), cudaMemcpyDeviceToHost, stream));
            RB_CUDA_TRY(cudaStreamSynchronize(stream));
            hsq = *hp;
            RB_CUDA_TRY(set_costs<In>(K, K0, hsq));
            h_pack_kernel<In, Real><<<tp, 256, 0, stream>>>(d, Hd.ptr, 1.0 / prm.scale, h.ptr);
            RB_CUDA_TRY(cudaGetLastError());
        }
        return setup_common();
    }

    // Everything after h: iterates, partial rows, tiles, cluster size.
    cudaError_t setup_common() {
        for (auto* b : {&xh, &x0, &r, &yh, &y0, &zh, &z0, &x2s, &dxs, &y2s, &z2s})
            RB_CUDA_TRY(b->alloc(nd, stream));
        tw = kXTile;
        const int ntc = (tp + tw - 1) / tw;
        const int ntc_low = (tp + kLowTW - 1) / kLowTW;
        nbx = n * ntc;
        nblo = n * ntc_low;
        x_smem = size_t(tw) * size_t(tp | 1) * sizeof(double);
        // z: a CTA of a cluster holds its rows of one period block (Tp - s
        // entries per row; z_task), or of a pair of blocks (Tp + 1 entries
        // per row; z_task_pair) in FP64 when the pairs still fill a wave of
        // two CTAs per SM.  Measured per solve: FP64 pairs are 6-14 % faster
        // at N = 10..200, T = 300..1000; in FP32 (two z CTAs per SM) and on
        // grids under a wave, pairs are 1-7 % slower.
        auto cluster_for = [&](int row) {
            int c = 1;
            while (c < kMaxCluster && size_t((n + c - 1) / c) * row * sizeof(Real) > size_t(z_slice_bytes<Real>())) ++c;
            return c > n ? n : c;
        };
        int zrow = tp + 1, csize = cluster_for(tp + 1);
        {
            int dev = 0, sms = 0;
            RB_CUDA_TRY(cudaGetDevice(&dev));
            RB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            d.zpair = sizeof(Real) == 8 && (long long)(tp / 2) * csize >= 2LL * sms ? 1 : 0;
            // REFORM_PRIA_ZPAIR=0|1 overrides the choice (tests, measurements)
            const char* env = std::getenv("REFORM_PRIA_ZPAIR");
            if (env && (env[0] == '0' || env[0] == '1') && env[1] == '\0') d.zpair = env[0] - '0';
        }
        if (!d.zpair) {
            zrow = tp;
            csize = cluster_for(tp);
        }
        yz_smem = size_t((n + csize - 1) / csize) * zrow * sizeof(Real);
        d.zstaged = 1;
        if (yz_smem > size_t(z_slice_bytes<Real>())) {   // the largest block exceeds a full cluster's slices
            d.zstaged = 0;
            yz_smem = 0;
        }
        nbyz = tp * csize;
        nby = int(((long long)tp * n + kYThreads / 32 - 1) / (kYThreads / 32));
        RB_CUDA_TRY(px.alloc(size_t(nbx) * 2, stream));
        RB_CUDA_TRY(pyz.alloc(size_t(nbyz) * 3, stream));
        RB_CUDA_TRY(py.alloc(size_t(nby) * 3, stream));
        RB_CUDA_TRY(pup.alloc(size_t(tp) * 3, stream));
        RB_CUDA_TRY(plo.alloc(size_t(nblo), stream));
        RB_CUDA_TRY(final_up.alloc(size_t(tp) * 3, stream));
        RB_CUDA_TRY(thx.alloc(size_t(n) * tp, stream));
        RB_CUDA_TRY(thy.alloc(size_t(n) * tp, stream));
        RB_CUDA_TRY(thz.alloc(size_t(tp), stream));
        RB_CUDA_TRY(ctl.alloc(1, stream));
        for (auto& ev : done) RB_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        d.ntc = ntc;
        d.ntc_low = ntc_low;
        d.csize = csize;
        d.eta = p.eta;
        d.h = h.ptr;
        d.xh = xh.ptr; d.x0 = x0.ptr; d.r = r.ptr; d.yh = yh.ptr; d.y0 = y0.ptr; d.zh = zh.ptr; d.z0 = z0.ptr;
        d.x2s = x2s.ptr; d.dxs = dxs.ptr; d.y2s = y2s.ptr; d.z2s = z2s.ptr;
        d.px = px.ptr; d.py = py.ptr; d.pyz = pyz.ptr; d.pup = pup.ptr; d.plo = plo.ptr; d.ctl = ctl.ptr;
        d.thx = thx.ptr; d.thy = thy.ptr; d.thz = thz.ptr;
        prm.tolerance = p.tolerance;
        prm.eta = p.eta;
        prm.max_iter = p.max_iter;
        prm.op_steps = p.op_steps;
        prm.beta_sufficient = p.beta_sufficient;
        prm.beta_necessary = p.beta_necessary;
        prm.beta_artificial = p.beta_artificial;
        prm.theta_target = p.theta_target;
        prm.theta_decay = p.theta_decay;
        prm.vanilla_max = p.use_halpern ? (long long)p.op_steps * p.warm_steps : p.max_iter;
        prm.start_max = vanilla_phase() ? prm.vanilla_max : p.max_iter;
        prm.omega0 = p.omega;
        prm.vanilla_solve = p.use_halpern ? 0 : 1;
        RB_CUDA_TRY(set_attributes());
        block_nodes = 3LL * p.op_steps + 3 + 4;   // x, y, z per step; bounds, check; restart x, y, z, check
        RB_CUDA_TRY(init_mega());
        return cudaGetLastError();
    }

    // --- the persistent kernel -------------------------------------------
    // It needs every z task in one CTA (cluster size 1, single blocks, staged
    // in shared memory) and its dynamic shared memory (the largest of the x
    // tile, the y rows, the z block) within kMegaSmemLimit.
    bool mega_possible() const {
        return mega_grid > 0 && d.csize == 1 && !d.zpair && d.zstaged && mega_smem <= kMegaSmemLimit;
    }

    cudaError_t init_mega() {
        mega_smem = std::max({x_smem, size_t(kYThreads / 32) * tp * sizeof(Real), yz_smem});
        mega_grid = 0;
        if (mega_smem <= kMegaSmemLimit) {
            int dev = 0, sms = 0, per_sm = 1 << 30;
            RB_CUDA_TRY(cudaGetDevice(&dev));
            RB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            for (auto fn : {mega_block_kernel<Real, false>, mega_block_kernel<Real, true>}) {
                int k = 0;   // (their shared-memory limit is set with the others, set_attributes)
                RB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, fn, kMegaThreads, mega_smem));
                per_sm = std::min(per_sm, k);
            }
            // no phase has more units than this: more CTAs would only wait
            const long long units = std::max({(long long)nbx, (long long)tp + nby, (long long)tp + nblo});
            mega_grid = int(std::min<long long>((long long)per_sm * sms, units));
        }
        // REFORM_PRIA_MEGA=0|1 sets the initial mode (tests, measurements);
        // REFORM_PRIA_MEGA_PHANTOM=k makes every barrier wait for k CTAs that
        // are never launched, so each wait runs out (the fault-injection test)
        const char* env = std::getenv("REFORM_PRIA_MEGA");
        int mode = -1;
        if (env && (env[0] == '0' || env[0] == '1') && env[1] == '\0') mode = env[0] - '0';
        const char* ph = std::getenv("REFORM_PRIA_MEGA_PHANTOM");
        if (ph) {
            mega_phantom = unsigned(std::strtoul(ph, nullptr, 10));
            if (mega_phantom) mega_wait_ns = 50000000ull;   // 50 ms: the test waits for every barrier
        }
        return set_mega(mode);
    }

    cudaError_t set_mega(int mode) {
        mega_mode = mode < 0 ? -1 : (mode ? 1 : 0);
        const bool want = mega_mode == 1 || (mega_mode < 0 && nd <= kMegaAutoEntries);
        mega = want && mega_possible();
        if (mega && !bar.ptr) {
            RB_CUDA_TRY(bar.alloc(1, stream));
            RB_CUDA_TRY(cudaMemsetAsync(bar.ptr, 0, sizeof(GridBar), stream));
        }
        return cudaSuccess;
    }

    cudaError_t launch_mega(bool vanilla) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(unsigned(mega_grid));
        cfg.blockDim = dim3(unsigned(kMegaThreads));
        cfg.dynamicSmemBytes = mega_smem;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;   // every CTA resident at once, or no launch
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const MegaArgs a{bar.ptr, unsigned(mega_grid) + mega_phantom, mega_wait_ns};
        if (vanilla) return cudaLaunchKernelEx(&cfg, mega_block_kernel<Real, true>, d, prm, a);
        return cudaLaunchKernelEx(&cfg, mega_block_kernel<Real, false>, d, prm, a);
    }

    // The dynamic shared-memory limit is a property of the kernel, shared by
    // every solver in the process, so it is set to the most any instance can
    // ask for (x: a tile of the widest padded row; y/z: one cluster slice),
    // never to this instance's own need: a later, smaller instance must not
    // lower the limit under an earlier, larger one.
    template <int TW, bool R, bool C>
    static cudaError_t x_attr() {
        return cudaFuncSetAttribute(x_kernel<Real, TW, R, C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(x_smem_limit()));
    }
    template <bool R, bool C>
    static cudaError_t yz_attr() {
        RB_CUDA_TRY(cudaFuncSetAttribute(y_kernel<Real, R, C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(y_smem_limit())));
        for (auto fn : {z_entry<Real, z_threads<Real>(), R, C, false>(), z_entry<Real, z_threads<Real>(), R, C, true>()}) {
            RB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, z_slice_bytes<Real>()));
            RB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        }
        return cudaSuccess;
    }
    cudaError_t set_attributes() {
        if (x_smem > x_smem_limit()) return cudaErrorInvalidValue;
        int done = 0;   // the limits are the kernels': set once per process and device
        return once_per_device(&done, [](int* v) {
            RB_CUDA_TRY((x_attr<kXTile, true, false>()));
            RB_CUDA_TRY((x_attr<kXTile, true, true>()));
            RB_CUDA_TRY((x_attr<kXTile, false, true>()));
            RB_CUDA_TRY(cudaFuncSetAttribute(project_x_kernel<Real, kXTile>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(x_smem_limit())));
            RB_CUDA_TRY((yz_attr<true, false>()));
            RB_CUDA_TRY((yz_attr<true, true>()));
            RB_CUDA_TRY((yz_attr<false, true>()));
            RB_CUDA_TRY((x_attr<kXTile, false, false>()));
            RB_CUDA_TRY((yz_attr<false, false>()));
            for (auto fn : {mega_block_kernel<Real, false>, mega_block_kernel<Real, true>})
                RB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kMegaSmemLimit)));
            *v = 1;
            return cudaSuccess;
        });
    }

    // Plain PDHG: the whole solve without Halpern, or warm_steps check blocks
    // before it (solver.py:601-606, 680-694).
    bool vanilla_phase() const { return !p.use_halpern || p.warm_steps > 0; }

    template <bool R, bool C>
    cudaError_t launch_x(const Real* xs, const Real* ys, const Real* zs, int step, int gate,
                         cudaStream_t on = nullptr) {
        x_kernel<Real, kXTile, R, C><<<n * d.ntc, kXThreads, x_smem, on ? on : stream>>>(d, xs, ys, zs, step, gate);
        return cudaGetLastError();
    }

    template <bool R, bool C>
    // the y half-step (one warp per row) and then the z half-step (a cluster
    // per z task: a period block, or a pair of them); two launches
    cudaError_t launch_yz(const Real* ys, const Real* zs, int step, int gate, cudaStream_t on = nullptr) {
        cudaStream_t st = on ? on : stream;
        y_kernel<Real, R, C><<<nby, kYThreads, size_t(kYThreads / 32) * tp * sizeof(Real), st>>>(d, ys, step, gate);
        RB_CUDA_TRY(cudaGetLastError());
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(unsigned(z_tasks() * d.csize));   // a cluster per z task
        cfg.blockDim = dim3(z_threads<Real>());
        cfg.dynamicSmemBytes = yz_smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = unsigned(d.csize);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if (d.zpair) return cudaLaunchKernelEx(&cfg, z_entry<Real, z_threads<Real>(), R, C, true>(), d, zs, step, gate);
        return cudaLaunchKernelEx(&cfg, z_entry<Real, z_threads<Real>(), R, C, false>(), d, zs, step, gate);
    }

    cudaError_t launch_check(int mode) {
        check_kernel<<<1, kCheckBlock, 0, stream>>>(d.ctl, prm, d.px, nbx, d.py, nby, d.pyz, nbyz, d.pup, tp, d.plo,
                                                   nblo, mode);
        return cudaGetLastError();
    }

    // --- profiling ------------------------------------------------------
    static constexpr int kKinds = 9;   // x, yz, x and yz at the check, upper, lower, check, restart; a mega block
    std::vector<cudaEvent_t> evpool;
    std::vector<std::pair<int, int>> marks;
    bool profiling = false;
    cudaError_t mark_begin(int kind) {
        if (!profiling) return cudaSuccess;
        const int idx = int(marks.size()) * 2;
        while (int(evpool.size()) < idx + 2) {
            cudaEvent_t ev;
            RB_CUDA_TRY(cudaEventCreate(&ev));
            evpool.push_back(ev);
        }
        marks.emplace_back(kind, idx);
        return cudaEventRecord(evpool[idx], stream);
    }
    cudaError_t mark_end() {
        if (!profiling) return cudaSuccess;
        return cudaEventRecord(evpool[marks.back().second + 1], stream);
    }
#define RB_PTIMED(kind, expr)            \
    do {                                 \
        RB_CUDA_TRY(mark_begin(kind));   \
        RB_CUDA_TRY(expr);               \
        RB_CUDA_TRY(mark_end());         \
    } while (0)

    cudaError_t enqueue_block() {
        if (mega) {
            RB_PTIMED(8, launch_mega(false));
            return cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream);
        }
        const int op = p.op_steps;
        for (int s = 0; s < op; ++s) {
            if (s + 1 < op) {
                RB_PTIMED(0, (launch_x<true, false>(d.xh, d.yh, d.zh, s, 0)));
                RB_PTIMED(1, (launch_yz<true, false>(d.yh, d.zh, s, 0)));
            } else {
                RB_PTIMED(2, (launch_x<true, true>(d.xh, d.yh, d.zh, s, 0)));
                RB_PTIMED(3, (launch_yz<true, true>(d.yh, d.zh, s, 0)));
            }
        }
        RB_PTIMED(4, (upper_kernel<Real><<<tp, kAuxThreads, 0, stream>>>(d, d.x2s, tp, 0), cudaGetLastError()));
        RB_PTIMED(5, (lower_kernel<Real><<<nblo, kAuxThreads, 0, stream>>>(d, d.y2s, d.z2s), cudaGetLastError()));
        RB_PTIMED(6, launch_check(1));
        RB_PTIMED(7, (launch_x<false, true>(d.x2s, d.y2s, d.z2s, 0, 1)));
        RB_PTIMED(7, (launch_yz<false, true>(d.y2s, d.z2s, 0, 1)));
        RB_PTIMED(7, launch_check(2));
        RB_CUDA_TRY(cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream));
        return cudaGetLastError();
    }

    // The repeated runs' check block as one graph: block_gate_kernel, then a
    // conditional node whose body is the captured block, so a block launched
    // after termination skips its body on the device.  Where the conditional
    // graph cannot be built, the plain captured block (its kernels gated
    // one by one).
    cudaError_t capture_block() {
        gated = capture_gated_block() == cudaSuccess;
        if (gated) return cudaSuccess;
        (void)cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        RB_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t st = enqueue_block();
        cudaError_t st2 = cudaStreamEndCapture(stream, &graph);
        RB_CUDA_TRY(st);
        RB_CUDA_TRY(st2);
        return cudaGraphInstantiate(&exec, graph, 0);
    }

    cudaError_t capture_gated_block() {
        RB_CUDA_TRY(cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle handle;
        RB_CUDA_TRY(cudaGraphConditionalHandleCreate(&handle, graph, 0, cudaGraphCondAssignDefault));
        cudaGraphNode_t gate;
        cudaKernelNodeParams kp = {};
        void* args[2] = {&d.ctl, &handle};
        kp.func = reinterpret_cast<void*>(block_gate_kernel);
        kp.gridDim = dim3(1);
        kp.blockDim = dim3(32);
        kp.kernelParams = args;
        RB_CUDA_TRY(cudaGraphAddKernelNode(&gate, graph, nullptr, 0, &kp));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        cudaGraphNode_t cond;
        RB_CUDA_TRY(cudaGraphAddNode(&cond, graph, &gate, 1, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        RB_CUDA_TRY(cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        cudaError_t st = enqueue_block();
        cudaGraph_t captured = nullptr;
        cudaError_t st2 = cudaStreamEndCapture(stream, &captured);
        RB_CUDA_TRY(st);
        RB_CUDA_TRY(st2);
        return cudaGraphInstantiate(&exec, graph, 0);
    }

    cudaError_t launch_block() { return exec && !mega ? cudaGraphLaunch(exec, stream) : enqueue_block(); }
    long long block_launches() const { return mega ? 1 : block_nodes + (exec && gated ? 1 : 0); }
    // the error of a block whose grid barrier ran out (the persistent kernel)
    static constexpr int kMegaWaitError = int(cudaErrorLaunchTimeout);

    int set_megakernel(int mode, int* active) override {
        const cudaError_t st = set_mega(mode);
        if (active) *active = mega ? 1 : 0;
        return int(st);
    }

    // The trace ring lives in the check parameters, which a captured block
    // holds by value: a new ring drops the capture, the next run makes one.
    int set_trace(int capacity) override {
        RB_CUDA_TRY(cudaStreamSynchronize(stream));
        trace.release();
        prm.trace = nullptr;
        prm.trace_cap = 0;
        if (capacity > 0) {
            RB_CUDA_TRY(trace.alloc(size_t(capacity), stream));
            prm.trace = trace.ptr;
            prm.trace_cap = capacity;
        }
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        return 0;
    }

    // The last run's records, oldest first: min(written, ring, capacity) of
    // them, the most recent; *total = records written.
    int get_trace(reform_trace_record* out, int capacity, int64_t* total) override {
        const long long len = std::max(0LL, mirror->trace_len);
        if (total) *total = len;
        if (!prm.trace || !out || capacity <= 0) return 0;
        std::vector<reform_trace_record> ring(size_t(prm.trace_cap));
        RB_CUDA_TRY(cudaMemcpyAsync(ring.data(), prm.trace, sizeof(reform_trace_record) * ring.size(),
                                    cudaMemcpyDeviceToHost, stream));
        RB_CUDA_TRY(cudaStreamSynchronize(stream));
        const long long count = std::min<long long>({len, (long long)prm.trace_cap, (long long)capacity});
        for (long long k = 0; k < count; ++k) out[k] = ring[size_t((len - count + k) % prm.trace_cap)];
        return 0;
    }

    int set_warm(const double* wx, const double* wy, const double* wz) override {
        if (!wx || !wy || !wz) {
            has_warm = false;
            return 0;
        }
        const size_t full = size_t(n) * t * t;
        if (warm[0].upload(wx, full, stream) || warm[1].upload(wy, full, stream) ||
            warm[2].upload(wz, full, stream) || cudaStreamSynchronize(stream))
            return int(cudaErrorMemoryAllocation);
        has_warm = true;
        return 0;
    }

    cudaError_t start_solve() {
        nlaunch = 0;
        if (mega) RB_CUDA_TRY(cudaMemsetAsync(bar.ptr, 0, sizeof(GridBar), stream));
        // every run starts its thresholds cold (all-NaN bytes)
        RB_CUDA_TRY(cudaMemsetAsync(thx.ptr, 0xFF, sizeof(double) * thx.count, stream));
        RB_CUDA_TRY(cudaMemsetAsync(thy.ptr, 0xFF, sizeof(double) * thy.count, stream));
        RB_CUDA_TRY(cudaMemsetAsync(thz.ptr, 0xFF, sizeof(double) * thz.count, stream));
        init_kernel<Real><<<tp, 256, 0, stream>>>(d, d.ctl, p.omega, p.theta_initial);
        nlaunch += 1;
        if (has_warm) {
            warm_pack_kernel<Real><<<tp, 256, 0, stream>>>(d, warm[0].ptr, warm[1].ptr, warm[2].ptr, d.x0, d.y0,
                                                           d.z0);
            project_x_kernel<Real, kXTile><<<n * d.ntc, kXThreads, x_smem, stream>>>(d, d.x0);
            project_yz_kernel<Real><<<tp, kAuxThreads, 0, stream>>>(d, d.y0, d.z0);
            nlaunch += 3;
        }
        // x1 = raw_step(x0): one vanilla step from the start point, with the
        // sums for the error, and the bounds at the start point itself.
        RB_CUDA_TRY(cudaGetLastError());
        upper_kernel<Real><<<tp, kAuxThreads, 0, stream>>>(d, d.x0, tp, 0);
        lower_kernel<Real><<<nblo, kAuxThreads, 0, stream>>>(d, d.y0, d.z0);
        RB_CUDA_TRY((launch_x<false, true>(d.x0, d.y0, d.z0, 0, 0)));
        RB_CUDA_TRY((launch_yz<false, true>(d.y0, d.z0, 0, 0)));
        RB_CUDA_TRY(launch_check(0));
        RB_CUDA_TRY(cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream));
        nlaunch += 6;
        return cudaStreamSynchronize(stream);
    }

    // One check block of the vanilla phase: op_steps plain steps of the
    // current point in place, then the bounds at it and the check (mode 3).
    cudaError_t enqueue_vanilla_block() {
        if (mega) {
            RB_CUDA_TRY(launch_mega(true));
            nlaunch += 1;
            return cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream);
        }
        for (int s = 0; s < p.op_steps; ++s) {
            RB_CUDA_TRY((launch_x<false, false>(d.xh, d.yh, d.zh, 0, kGateVanilla)));
            RB_CUDA_TRY((launch_yz<false, false>(d.yh, d.zh, 0, kGateVanilla)));
        }
        upper_kernel<Real><<<tp, kAuxThreads, 0, stream>>>(d, d.xh, tp, 0);
        lower_kernel<Real><<<nblo, kAuxThreads, 0, stream>>>(d, d.yh, d.zh);
        RB_CUDA_TRY(launch_check(3));
        nlaunch += 3LL * p.op_steps + 3;
        return cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream);
    }

    // The vanilla phase from the start point (x0, the anchor, is kept for
    // the drift that sets omega), then, for the Halpern method, the step
    // that makes the current point the anchor (mode 4).
    // Seconds since `started`, against the budget.
    bool over_budget(std::chrono::steady_clock::time_point started) const {
        return time_limit >= 0.0 &&
               std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count() > time_limit;
    }

    cudaError_t run_vanilla(std::chrono::steady_clock::time_point started, bool& timed_out) {
        const size_t bytes = sizeof(Real) * size_t(nd);
        RB_CUDA_TRY(cudaMemcpyAsync(d.xh, d.x0, bytes, cudaMemcpyDeviceToDevice, stream));
        RB_CUDA_TRY(cudaMemcpyAsync(d.yh, d.y0, bytes, cudaMemcpyDeviceToDevice, stream));
        RB_CUDA_TRY(cudaMemcpyAsync(d.zh, d.z0, bytes, cudaMemcpyDeviceToDevice, stream));
        for (;;) {
            RB_CUDA_TRY(enqueue_vanilla_block());
            RB_CUDA_TRY(cudaStreamSynchronize(stream));
            if (mirror->status) return cudaErrorLaunchTimeout;
            if (mirror->terminated || mirror->phase_done) break;
            if (over_budget(started)) {
                timed_out = true;        // the last check's point: the current one (slot 3)
                return cudaSuccess;
            }
            if (p.verbose)
                fprintf(stderr, "pria: iter %8lld  primal %.9e  dual %.9e  gap %.3e  (vanilla)\n",
                        mirror->iteration, mirror->upper, mirror->lower, mirror->gap);
        }
        if (mirror->terminated || !p.use_halpern) return cudaSuccess;
        RB_CUDA_TRY((launch_x<false, true>(d.xh, d.yh, d.zh, 0, kGateDrift)));
        RB_CUDA_TRY((launch_yz<false, true>(d.yh, d.zh, 0, kGateDrift)));
        RB_CUDA_TRY(launch_check(4));
        nlaunch += 4;
        RB_CUDA_TRY(cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream));
        return cudaStreamSynchronize(stream);
    }

    int run() override {
        const auto started = std::chrono::steady_clock::now();
        bool timed_out = false;
        if (runs++ > 0 && !exec && !mega && p.use_halpern && capture_block() != cudaSuccess)
            return int(cudaErrorUnknown);
        cudaError_t st = start_solve();
        if (st != cudaSuccess) return int(st);
        if (!mirror->terminated && vanilla_phase() && (st = run_vanilla(started, timed_out)) != cudaSuccess)
            return mirror->status == kBoundsStatus ? kStatusBounds : int(st);
        if (timed_out && !mirror->terminated) return kStatusTimeLimit;
        if (!mirror->terminated) {
            for (int kk = 0; kk < 2; ++kk) {
                if ((st = launch_block()) != cudaSuccess) return int(st);
                if ((st = cudaEventRecord(done[kk], stream)) != cudaSuccess) return int(st);
                nlaunch += block_launches();
            }
            int kk = 0;
            for (;;) {
                if ((st = cudaEventSynchronize(done[kk])) != cudaSuccess) return int(st);
                if (mirror->terminated && !mirror->status && exec && gated && !mega)
                    nlaunch -= block_nodes;   // the block behind it ran its gate alone
                if (mirror->status || mirror->terminated) break;
                if (p.verbose)
                    fprintf(stderr, "pria: iter %8lld  primal %.9e  dual %.9e  gap %.3e  omega %.3e\n",
                            mirror->iteration, mirror->upper, mirror->lower, mirror->gap, mirror->omega);
                if (over_budget(started)) {
                    timed_out = true;
                    break;
                }
                if ((st = launch_block()) != cudaSuccess) return int(st);
                if ((st = cudaEventRecord(done[kk], stream)) != cudaSuccess) return int(st);
                nlaunch += block_launches();
                kk ^= 1;
            }
        }
        // The block still in flight after a time-out finishes (its check
        // included) before the mirror is read back; the result is the point and
        // bracket of the last check it completed.
        if ((st = cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
            (st = cudaStreamSynchronize(stream)) != cudaSuccess)
            return int(st);
        if (mirror->status == kBoundsStatus) return kStatusBounds;
        if (mirror->status) return kMegaWaitError;
        return timed_out && !mirror->terminated ? kStatusTimeLimit : 0;
    }

    int run_profiled(double* ms, long long* count) override {
        for (int kk = 0; kk < kKinds; ++kk) { ms[kk] = 0.0; count[kk] = 0; }
        cudaError_t st = start_solve();
        if (st != cudaSuccess) return int(st);
        // the vanilla phase, if any, runs untimed: the kinds are the Halpern block's
        bool timed_out = false;   // no budget here: time_limit is not consulted by a profiled run
        const auto never = std::chrono::steady_clock::now();
        const double budget = time_limit;
        time_limit = -1.0;
        st = !mirror->terminated && vanilla_phase() ? run_vanilla(never, timed_out) : cudaSuccess;
        time_limit = budget;
        if (st != cudaSuccess) return int(st);
        profiling = true;
        while (!mirror->terminated) {
            marks.clear();
            if ((st = enqueue_block()) != cudaSuccess || (st = cudaStreamSynchronize(stream)) != cudaSuccess) {
                profiling = false;
                return int(st);
            }
            nlaunch += block_launches();
            if (mirror->status) {
                profiling = false;
                return kMegaWaitError;
            }
            for (auto& mk : marks) {
                float tm = 0.f;
                if ((st = cudaEventElapsedTime(&tm, evpool[mk.second], evpool[mk.second + 1])) != cudaSuccess) {
                    profiling = false;
                    return int(st);
                }
                ms[mk.first] += tm;
                count[mk.first] += 1;
            }
        }
        profiling = false;
        if ((st = cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
            (st = cudaStreamSynchronize(stream)) != cudaSuccess)
            return int(st);
        return 0;
    }

    // The objective at the returned (unpadded) x, in instance units.
    cudaError_t final_primal(double* out) {
        const Real* xs = point(0);
        Dev<Real> dd = d;
        dd.pup = final_up.ptr;
        upper_kernel<Real><<<tp, kAuxThreads, 0, stream>>>(dd, xs, t, 1);
        std::vector<double> host(size_t(tp) * 3);
        RB_CUDA_TRY(cudaMemcpyAsync(host.data(), final_up.ptr, sizeof(double) * host.size(),
                                    cudaMemcpyDeviceToHost, stream));
        RB_CUDA_TRY(cudaStreamSynchronize(stream));
        double sum = 0.0;
        for (double v : host) sum += v;
        *out = sum * prm.scale;
        return cudaSuccess;
    }

    template <class Out>
    cudaError_t unpack(const Real* src, int mode, Out* host) {
        PoolBuf<Out> buf;
        const size_t full = size_t(n) * t * t;
        RB_CUDA_TRY(buf.alloc(full, stream));
        unpack_kernel<Real, Out><<<1184, 256, 0, stream>>>(d, src, mode, buf.ptr);
        // A large output goes through the library's pinned ring: the copy
        // engine fills it at the pinned rate (55 GB/s against 20 pageable)
        // while the host threads move the other slot into the caller's
        // memory, whose first-touch page faults then run on several threads
        // (N = 100, T = 500: 127 -> 52 ms for the three FP32 outputs).  A
        // small one goes by the driver's pageable copy, which is cheaper
        // there (N = 30, T = 75, 1.35 MB an output: 0.13 against 0.26 ms).
        constexpr size_t kRingBytes = size_t(16) << 20;
        if (sizeof(Out) * full >= kRingBytes) {
            const cudaError_t st = staged_download(host, buf.ptr, sizeof(Out) * full, stream);
            if (st != cudaErrorMemoryAllocation) return st;   // no ring to be had: the driver's copy
        }
        RB_CUDA_TRY(cudaMemcpyAsync(host, buf.ptr, sizeof(Out) * full, cudaMemcpyDeviceToHost, stream));
        return cudaStreamSynchronize(stream);
    }

    // The returned point: 1 the anchor (the start, or the point the vanilla
    // phase ended at), 2 the step at the last check, 3 the current point of
    // a vanilla solve.  k = 0, 1, 2 for x, y, z.
    const Real* point(int k) const {
        const int slot = mirror->result_slot;
        const Real* const anchor[3] = {d.x0, d.y0, d.z0};
        const Real* const step[3] = {d.x2s, d.y2s, d.z2s};
        const Real* const cur[3] = {d.xh, d.yh, d.zh};
        return slot == 1 ? anchor[k] : slot == 3 ? cur[k] : step[k];
    }

    template <class Out>
    int result_t(Out* x, Out* y, Out* z, pria_result_info* info) {
        const Real* xs = point(0);
        const Real* ys = point(1);
        const Real* zs = point(2);
        cudaError_t st;
        if (x && (st = unpack<Out>(xs, 0, x)) != cudaSuccess) return int(st);
        if (y && (st = unpack<Out>(ys, 1, y)) != cudaSuccess) return int(st);
        if (z && (st = unpack<Out>(zs, 2, z)) != cudaSuccess) return int(st);
        if (info) {
            double primal = 0.0;
            if ((st = final_primal(&primal)) != cudaSuccess) return int(st);
            info->iterations = mirror->iteration;
            info->primal_objective = primal;
            info->dual_objective = mirror->lower;
            info->relative_gap = (primal - mirror->lower) / (1.0 + std::fabs(primal) + std::fabs(mirror->lower));
        }
        return 0;
    }
    int result(double* x, double* y, double* z, pria_result_info* info) override {
        return result_t<double>(x, y, z, info);
    }
    int result_f32(float* x, float* y, float* z, pria_result_info* info) override {
        return result_t<float>(x, y, z, info);
    }

    long long launches() const override { return nlaunch; }

    size_t device_bytes() const {
        size_t b = 0;
        for (auto* x : {&h, &k, &xh, &x0, &r, &yh, &y0, &zh, &z0, &x2s, &dxs, &y2s, &z2s})
            b += x->count * sizeof(Real);
        for (auto* x : {&px, &py, &pyz, &pup, &plo, &final_up, &thx, &thy, &thz}) b += x->count * sizeof(double);
        return b + sizeof(Control);
    }
};

template <class In>
static int create(int64_t n, int64_t t, const In* K, double K0, const In* H, const pria_params* params,
                  int use_float32, cudaStream_t stream, std::unique_ptr<SolverBase>& out) {
    if (n < 1 || t < 1 || !K || !H || !params) return int(cudaErrorInvalidValue);
    const int64_t tp = t + (t & 1);
    if (tp > kMaxPeriods || n > (1LL << 24)) return int(cudaErrorInvalidValue);
    pria_params p = *params;
    if (p.op_steps < 2) p.op_steps = 2;
    if (p.warm_steps < 0) p.warm_steps = 0;
    if (p.max_iter < 0) p.max_iter = -1;
    cudaError_t st;
    if (use_float32) {
        auto* s = new Solver<float>();
        out.reset(s);
        s->p = p;
        st = s->template setup<In>(n, t, K, K0, H, stream);
    } else {
        auto* s = new Solver<double>();
        out.reset(s);
        s->p = p;
        st = s->template setup<In>(n, t, K, K0, H, stream);
    }
    return int(st);
}

static int create_demand(int64_t n, int64_t t, const double* K, double K0, const double* rate,
                         const double* demand, const pria_params* params, int use_float32, cudaStream_t stream,
                         std::unique_ptr<SolverBase>& out) {
    if (n < 1 || t < 1 || !K || !rate || !demand || !params) return int(cudaErrorInvalidValue);
    const int64_t tp = t + (t & 1);
    if (tp > kMaxPeriods || n > (1LL << 24)) return int(cudaErrorInvalidValue);
    pria_params p = *params;
    if (p.op_steps < 2) p.op_steps = 2;
    if (p.warm_steps < 0) p.warm_steps = 0;
    if (p.max_iter < 0) p.max_iter = -1;
    cudaError_t st;
    if (use_float32) {
        auto* s = new Solver<float>();
        out.reset(s);
        s->p = p;
        st = s->setup_demand(n, t, K, K0, rate, demand, stream);
    } else {
        auto* s = new Solver<double>();
        out.reset(s);
        s->p = p;
        st = s->setup_demand(n, t, K, K0, rate, demand, stream);
    }
    return int(st);
}

}  // namespace
}  // namespace pria
}  // namespace rb200
