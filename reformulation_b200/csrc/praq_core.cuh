// praq_core.cuh -- PRAQ (QUBO roof-dual LP) on B200: restarted, reflected
// Halpern PDHG on the half-edge lift, FP64 or FP32 iterates with FP64
// reductions, restart logic and bounds.
//
// The algorithm is the reference's (qubo/praq-jax/praq/solver.py, the
// specification; qubo/praq-cuda/src/solver.cuh, its CUDA port).  The device
// design is this file's own:
//
// * ONE REAL PER EDGE for the dual.  Each edge's dual set is a segment of a
//   line: covering edges (W_ij > 0) live on {(mu, mu) : -w <= mu <= 0},
//   packing edges on {(a, w - a) : 0 <= a <= w} (projection.py:16-42).  The
//   Halpern combination is affine with weights summing to one, so every
//   iterate (projected or combined) stays on that line, and the pair is
//   carried as one coordinate u (mu, or a).  The projection of
//   y + eta omega (q - S r) then collapses to
//       covering:  mu' = clip(mu + (eta omega / 2)(1 - r_i - r_j), -w, 0)
//       packing:   a'  = clip(a  + (eta omega / 2)(r_j - r_i),      0, w)
// * SLOT 1 PUSHED OR PULLED.  Edges are sorted by first end (stable), so a
//   node's first-end half-edges are one run of `pred` (slot 0 = u).  Each
//   edge's slot-1 value (u, or w - u) must reach its second end too, through
//   one random access per edge, which can sit on either side:
//   push: the edge kernel writes it to `pred1` at the edge's position in
//   second-end order (`colpos`), and the node kernel reads its second-end
//   half-edges as one coalesced run;
//   pull: the edge kernel writes it to `pred1` in edge order (coalesced), and
//   the node kernel gathers it through `colidx` (the edges in second-end
//   order).
//   While the edge arrays sit in L2 the scattered write is cheap and the
//   latency-bound node kernel should not wait on a dependent gather, so push
//   wins (n = 1e5, m = 1e6: 1.50 vs 1.54 ms per solve); once they spill to
//   DRAM every scattered 4-byte write costs a sector read and write, and pull
//   wins (n = 2e6, m = 2e7: 21.9 vs 33.1 ms).  The solver pulls when the edge
//   arrays exceed twice the L2 size.
// * `pred`/`pred1` hold the NEXT step's Halpern-combined dual, computed by the
//   edge kernel as it finishes a step (as the reference does), so a reflected
//   step streams one real per edge of dual state plus the anchor.
// * Every decision of _halpern_step (restart tests, omega/theta update,
//   termination) runs on the device in `check_kernel`; one op_steps block
//   (op_steps x (node, edge), lower-bound pass, check, the gated restart step)
//   needs no host input, so repeated runs replay it as a captured CUDA graph.
//   The host keeps one block in flight ahead of the one it inspects.
// * The instance is laid out ON THE DEVICE from the caller's COO arrays:
//   validation, scaling, the stable sorts by first and second end (CUB radix
//   sort; the first is skipped when the input is already sorted by first end),
//   the run pointers and degrees are kernels, so a one-shot solve pays one
//   upload of the raw arrays and no O(m) host work.
//
// Determinism: every sum has a fixed order that depends on the instance and
// the launch shape only, so runs are bitwise reproducible.
#pragma once

#include "../../include/praq.h"
#include "common.cuh"
#include "memory.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <memory>

namespace rb200 {
namespace praq {
namespace {

constexpr double kEta = 0.999;   // 0.999 / ||A||_2, ||A||_2 = 1 for the half-edge lift
constexpr int kBlock = 256;
#ifndef RB200_PRAQ_EDGES_PER_THREAD
#define RB200_PRAQ_EDGES_PER_THREAD 4   // compile-time tunable (sweeps build with -D)
#endif
constexpr int kEdgesPerThread = RB200_PRAQ_EDGES_PER_THREAD;
// The steps without check sums have no per-tile results, so their edge grid
// may be cut differently from the check steps': FP32 iterates in the push
// layout (edge arrays in L2) take two edges a thread, twice the CTAs, which
// measured 2.6 % faster on the whole solve at n = 1e5, m = 1e6 than four (one:
// 0.6 %); FP64 iterates there, and the pull layout (edge arrays streamed from
// HBM), keep four (two: FP64 3 % slower at n = 1e5; FP32 1.3 % slower at
// n = 2e6, m = 2e7).
#ifndef RB200_PRAQ_PUSH_EDGES_PER_THREAD_F32
#define RB200_PRAQ_PUSH_EDGES_PER_THREAD_F32 2
#endif
template <class Real, bool Pull>
constexpr int plain_edges_per_thread() {
    return !Pull && sizeof(Real) == 4 ? RB200_PRAQ_PUSH_EDGES_PER_THREAD_F32 : kEdgesPerThread;
}
constexpr int kNodeSums = 3;     // sum deg (x1-x2)^2, sum deg (x1-x0)^2, sum d . bx
constexpr int kEdgeSums = 5;     // sum |y1-y2|^2, <S(x1-x2), y1-y2>, sum |y1-y0|^2,
                                 // upper edge term at bx, sum of covering by_1
constexpr int kCheckBlock = 256;
constexpr int kPrepBlocks = 296; // fixed grid of the preprocessing reduction
constexpr int64_t kHostCheckEdges = 16384;   // up to this many edges the set-up checks the input on the host

// Scalar state of the solve (StepArguments' scalars, solver.py:229-256),
// resident on the device.
struct Control {
    double omega, theta, fp_error, check_error;
    double new_error, lower, upper, gap;
    long long restart_iter, iteration;
    int terminated;   // the loop is over
    int restart;      // the restart step of this block is pending
    int result_slot;  // 1: (x1, u0) hold the returned point, 2: (x2, u2s)
    int status;
    long long trace_len;   // convergence-trace records written this run
};
static_assert(sizeof(Control) <= 256, "a pinned mirror slot holds one Control");

struct Params {
    double tolerance;
    long long max_iter, op_steps;
    double beta_sufficient, beta_necessary, beta_artificial;
    double theta_target, theta_decay;
    reform_trace_record* trace;   // the convergence-trace ring (null: none)
    int trace_cap;
};

template <class Real>
struct alignas(16) Dev {   // (16-byte aligned: the batched engine copies descriptors in 16-byte pieces)
    int n, m;
    const int* row_ptr;    // [n+1] first-end runs in sorted edge order
    const int* col_ptr;    // [n+1] second-end runs in second-end order
    int pull;              // slot-1 layout: 1 pull (edge order), 0 push (second-end order)
    const int* colidx;     // [m] pull: the sorted edge at position k of second-end order
    const int* colpos;     // [m] push: the second-end position of sorted edge s
    const int2* ends;      // [m]
    const Real* w;         // [m] signed, 2 W_ij / scale
    const Real* diag;      // [n] W_ii / scale
    const Real* deg;       // [n] incident half-edges, floored at 1
    const double* scale;   // [1] objective scale
    Real *x1, *x2, *x0, *r;
    Real *pred, *pred1;    // next combined dual: slot 0 (sorted edge order) and slot 1 (by layout)
    Real *u0;              // anchor (sorted order)
    Real *u2s, *u2s1;      // y2 at the last check: slot 0 and slot 1, as pred and pred1
    double *pnode, *pedge, *plower;
    Control* ctl;
};

__device__ __forceinline__ bool skip(const Control* c, int gate) {
    return c->terminated || (gate && !c->restart);
}

#ifndef RB200_PRAQ_STAGE_BYTES
#define RB200_PRAQ_STAGE_BYTES 2048   // per warp, run and pass; compile-time tunable (sweeps build with -D)
#endif
#ifndef RB200_PRAQ_PULL
#define RB200_PRAQ_PULL 2   // slot-1 layout: 0 push, 1 pull, 2 by size
#endif
#ifndef RB200_PRAQ_GATHER
#define RB200_PRAQ_GATHER 2   // node gather: 0 one run after the other, 1 both at once, 2 by grid size
#endif
constexpr int kSeqChunk = 4;   // sequential gather: loads per lane in flight
constexpr int kGather = RB200_PRAQ_GATHER;
constexpr int kPull = RB200_PRAQ_PULL;
// half-edge values a warp stages per run and pass
template <class Real>
constexpr int stage_len() { return RB200_PRAQ_STAGE_BYTES / int(sizeof(Real)); }

// The sums of v over the runs [ptr[i], ptr[i+1]) of the 32 consecutive nodes
// i = base + lane of a warp, one node per lane.  The runs of consecutive nodes
// are adjacent, so the warp copies the whole range [ptr[base], ptr[base+32])
// through shared memory in coalesced passes of kStage values, and each lane
// adds its own run's part of every pass in order.  All lanes of the warp must
// call it (with the same base).  Few registers: the form for grids of many
// waves, where the issue rate, not the latency of one warp, bounds the kernel
// (chunks of 4 loads per lane: 2 % faster per solve at n >= 1.5e5 than an
// unrolled loop; 8 were no better).
template <class Real, class Acc, bool Indexed>
__device__ __forceinline__ Acc warp_runs(const int* __restrict__ ptr, const Real* v, const int* __restrict__ idx,
                                         int n, long long base, int lane, Real* __restrict__ stage, int m,
                                         int* status) {
    if (base >= n) return Acc(0);   // uniform over the warp
    const long long i = base + lane;
    const long long last = base + 32 < n ? base + 32 : n;
    const int lo_all = ptr[base], hi_all = ptr[last];
    // the warp's range, the same on every lane (the runs inside it follow)
    if (!index_ok(0 <= lo_all && lo_all <= hi_all && hi_all <= m, status)) return Acc(0);
    int a = 0, b = 0;
    if (i < n) {
        a = ptr[i];
        b = ptr[i + 1];
    }
    constexpr int kStage = stage_len<Real>();
    Acc s = Acc(0);
    for (int c0 = lo_all; c0 < hi_all; c0 += kStage) {
        const int c1 = min(hi_all, c0 + kStage);
        // chunks of kSeqChunk predicated loads per lane with no loop around
        // them: one round trip per chunk (an unrolled loop would end in a
        // remainder loop that waits for each load in turn)
        for (int k0 = c0; k0 < c1; k0 += 32 * kSeqChunk) {
            Real t[kSeqChunk];
            if constexpr (Indexed) {   // value k is v[idx[k]]
                int at[kSeqChunk];
#pragma unroll
                for (int u = 0; u < kSeqChunk; ++u) {
                    const int k = k0 + lane + 32 * u;
                    if (k < c1) at[u] = idx[k];
                }
#pragma unroll
                for (int u = 0; u < kSeqChunk; ++u) {
                    const int k = k0 + lane + 32 * u;
                    if (k < c1) t[u] = index_ok(unsigned(at[u]) < unsigned(m), status) ? v[at[u]] : Real(0);
                }
            } else {
#pragma unroll
                for (int u = 0; u < kSeqChunk; ++u) {
                    const int k = k0 + lane + 32 * u;
                    if (k < c1) t[u] = v[k];
                }
            }
#pragma unroll
            for (int u = 0; u < kSeqChunk; ++u) {
                const int k = k0 + lane + 32 * u;
                if (k < c1) stage[k - c0] = t[u];
            }
        }
        __syncwarp();
        const int lo = max(a, c0), hi = min(b, c1);
        for (int k = lo; k < hi; ++k) s += Acc(stage[k - c0]);
        __syncwarp();
    }
    return s;
}

// The sums, for the 32 consecutive nodes i = base + lane of a warp (one node
// per lane), of two runs at once: run a = va[pa[i] .. pa[i+1]) and run b =
// vb[k] (IndexB: vb[ib[k]]) for k in [pb[i], pb[i+1]).  The warp copies the
// ranges of both runs for its 32 nodes through shared memory in passes of
// kStage values each (run a and run b, or run b's indices, coalesced; with
// IndexB run b's values gathered), and every lane adds its own runs' parts of
// each pass in order.  A pass's loads, of both ranges, are predicated loads into registers
// with no loop around them, so all of them are in flight together: one memory
// round trip per pass (a warp-uniform exit skips the slots past both ranges).
// The sums are those of warp_runs, term for term and in the same order.
// Twice the registers of warp_runs: the form for grids of one wave, which the
// latency of a warp's dependent loads bounds.  All lanes of the warp must call
// it with the same base.
template <class Real, class Acc, bool IndexB>
__device__ __forceinline__ void warp_runs2(const int* __restrict__ pa, const Real* va, const int* __restrict__ pb,
                                           const Real* vb, const int* __restrict__ ib, int n, long long base, int lane,
                                           Real* __restrict__ sa,
                                           Real* __restrict__ sb, Acc& ra, Acc& rb, int m, int* status) {
    ra = Acc(0);
    rb = Acc(0);
    if (base >= n) return;   // uniform over the warp
    const long long i = base + lane;
    const long long last = base + 32 < n ? base + 32 : n;
    const int alo = pa[base], ahi = pa[last], blo = pb[base], bhi = pb[last];
    if (!index_ok(0 <= alo && alo <= ahi && ahi <= m && 0 <= blo && blo <= bhi && bhi <= m, status)) return;
    int a0 = 0, a1 = 0, b0 = 0, b1 = 0;
    if (i < n) {
        a0 = pa[i];
        a1 = pa[i + 1];
        b0 = pb[i];
        b1 = pb[i + 1];
    }
    constexpr int kStage = stage_len<Real>();
    constexpr int kPer = kStage / 32;
    static_assert(kStage % 32 == 0, "a pass is whole warp rows");
    for (int ca = alo, cb = blo; ca < ahi || cb < bhi; ca += kStage, cb += kStage) {
        const int ea = min(ahi, ca + kStage), eb = min(bhi, cb + kStage);
        // lane-relative bases and counts, so each load is a base plus an
        // immediate offset
        const Real* ga = va + (ca + lane);
        const int na = ea - ca - lane, nb = eb - cb - lane;
        const int wide = max(ea - ca, eb - cb);   // the same on every lane
        if constexpr (IndexB) {
            const int* __restrict__ gib = ib + (cb + lane);
            Real ta[kPer];
            int at[kPer];
#pragma unroll
            for (int q = 0; q < kPer; ++q) {
                if (32 * q >= wide) break;
                if (32 * q < na) ta[q] = ga[32 * q];
                if (32 * q < nb) at[q] = gib[32 * q];
            }
            // run a to shared memory first, so its registers are free before
            // the gather of run b is issued
#pragma unroll
            for (int q = 0; q < kPer; ++q) {
                if (32 * q >= wide) break;
                if (32 * q < na) sa[lane + 32 * q] = ta[q];
            }
#pragma unroll
            for (int q = 0; q < kPer; ++q) {
                if (32 * q >= wide) break;
                if (32 * q < nb) ta[q] = index_ok(unsigned(at[q]) < unsigned(m), status) ? vb[at[q]] : Real(0);
            }
#pragma unroll
            for (int q = 0; q < kPer; ++q) {
                if (32 * q >= wide) break;
                if (32 * q < nb) sb[lane + 32 * q] = ta[q];
            }
        } else {
            const Real* gb = vb + (cb + lane);
            Real ta[kPer], tb[kPer];
#pragma unroll
            for (int q = 0; q < kPer; ++q) {
                if (32 * q >= wide) break;
                if (32 * q < na) ta[q] = ga[32 * q];
                if (32 * q < nb) tb[q] = gb[32 * q];
            }
#pragma unroll
            for (int q = 0; q < kPer; ++q) {
                if (32 * q >= wide) break;
                if (32 * q < na) sa[lane + 32 * q] = ta[q];
                if (32 * q < nb) sb[lane + 32 * q] = tb[q];
            }
        }
        __syncwarp();
        for (int k = max(a0, ca), e = min(a1, ea); k < e; ++k) ra += Acc(sa[k - ca]);
        for (int k = max(b0, cb), e = min(b1, eb); k < e; ++k) rb += Acc(sb[k - cb]);
        __syncwarp();
    }
}

// S^T y at node base + lane: the node's run of `ys` (slot 0, first-end order)
// plus its run of slot-1 values of `yc`: in the push layout `yc` is in
// second-end order, in the pull layout it is in edge order and read through
// d.colidx (second-end order).  `stage` holds stage_runs<Wide> * stage_len
// values; all forms give the same sum.
template <bool Wide>
constexpr int stage_runs() { return Wide ? 2 : 1; }

// This warp's staging slice: one shared buffer per precision and width for
// every tile function of a kernel (the node step in its three forms and the
// lower-bound pass share it in the persistent kernel), runs * stage_len
// values per warp.
template <class Real, int Runs>
__device__ __forceinline__ Real* warp_stage() {
    __shared__ Real stage[kBlock / 32][Runs * stage_len<Real>()];
    return stage[threadIdx.x >> 5];
}

template <class Real, class Acc, bool Wide, bool Pull>
__device__ __forceinline__ Acc scatter_at(const Dev<Real>& d, const Real* ys, const Real* yc, long long base,
                                          int lane, Real* __restrict__ stage) {
    if constexpr (Wide) {
        Acc s0, s1;
        warp_runs2<Real, Acc, Pull>(d.row_ptr, ys, d.col_ptr, yc, d.colidx, d.n, base, lane, stage,
                                    stage + stage_len<Real>(), s0, s1, d.m, &d.ctl->status);
        return s0 + s1;
    } else {
        const Acc s0 = warp_runs<Real, Acc, false>(d.row_ptr, ys, nullptr, d.n, base, lane, stage, d.m, &d.ctl->status);
        const Acc s1 = warp_runs<Real, Acc, Pull>(d.col_ptr, yc, d.colidx, d.n, base, lane, stage, d.m, &d.ctl->status);
        return s0 + s1;
    }
}

// Primal half of one PDHG step, with the Halpern combination of x folded in
// (solver.py:259-267 and 276-292).  Reflect: x1 = lw (2 x2 - x1) + rw x0 with
// k = restart_iter + step + 1; vanilla: x1 = x2 and the anchor becomes x1.
// Check: the node sums of this step go to pnode.
template <class Real, bool Reflect, bool Check, bool Wide = false, bool Pull = false>
__device__ __forceinline__ void node_kernel_tile(const Dev<Real>& d, int tile, const Real* ys, const Real* yc, int step,
                                                 int bounds_at_1, int gate) {
    const Control* c = d.ctl;
    if (skip(c, gate)) return;
    __shared__ double scratch[kNodeSums * 32];
    Real* stage = warp_stage<Real, stage_runs<Wide>()>();
    const int lane = threadIdx.x & 31;
    const long long base = (long long)tile * blockDim.x + (threadIdx.x & ~31);
    const long long i = base + lane;
    const bool owner = i < d.n;
    // node data first, so its latency hides behind the gather
    Real x1o = Real(0), x2o = Real(0), x0o = Real(0), di = Real(0), dg = Real(1);
    if (owner) {
        x2o = d.x2[i];
        di = d.diag[i];
        dg = d.deg[i];
        if (Reflect) {
            x1o = d.x1[i];
            x0o = d.x0[i];
        }
    }
    const Real s = scatter_at<Real, Real, Wide, Pull>(d, ys, yc, base, lane, stage);
    double acc[kNodeSums] = {0.0, 0.0, 0.0};
    if (owner) {
        Real x1v;
        if (Reflect) {
            const double k = double(c->restart_iter + step + 1);
            const Real lw = Real(k / (k + 1.0)), rw = Real(1.0 / (k + 1.0));
            x1v = rfma(lw, rfma(Real(2), x2o, -x1o), rmul(rw, x0o));
        } else {
            x1v = x2o;
        }
        const Real ps = Real(kEta / c->omega);
        const Real x2v = clampv(rfma(-ps, (di - s) / dg, x1v), Real(0), Real(1));
        d.x1[i] = x1v;
        d.x2[i] = x2v;
        d.r[i] = rfma(Real(2), x2v, -x1v);
        if (!Reflect) d.x0[i] = x1v;
        if (Check) {
            const double dx = double(x1v) - double(x2v);
            const double dr = Reflect ? double(x1v) - double(x0o) : 0.0;
            acc[0] = double(dg) * dx * dx;
            acc[1] = double(dg) * dr * dr;
            acc[2] = double(di) * double(bounds_at_1 ? x1v : x2v);
        }
    }
    if (Check) {
        block_sums<kNodeSums>(acc, scratch, acc);
        if (threadIdx.x == 0) {
            for (int k = 0; k < kNodeSums; ++k) d.pnode[size_t(tile) * kNodeSums + k] = acc[k];
        }
    }
}

template <class Real, bool Reflect, bool Check, bool Wide = false, bool Pull = false>
__global__ void __launch_bounds__(kBlock)
node_kernel(Dev<Real> d, const Real* __restrict__ ys, const Real* __restrict__ yc, int step,
            int bounds_at_1, int gate) {
    pdl_wait();
    pdl_launch_dependents();
    node_kernel_tile<Real, Reflect, Check, Wide, Pull>(d, blockIdx.x, ys, yc, step, bounds_at_1, gate);
}

// Dual half of one PDHG step (solver.py:269-273, projection.py:16-42) in the
// one-coordinate form, plus the prediction of the next step's combined dual.
// Each thread takes kEdgesPerThread edges a block-stride apart, so all their
// loads are in flight together.
template <class Real, bool Reflect, bool Check, bool Pull = false, int EPT = kEdgesPerThread>
__device__ __forceinline__ void edge_kernel_tile(const Dev<Real>& d, int tile, const Real* ysrc, int step, int bounds_at_1, int gate) {
    const Control* c = d.ctl;
    if (skip(c, gate)) return;
    __shared__ double scratch[kEdgeSums * 32];
    const int base = tile * (kBlock * EPT) + threadIdx.x;
    const Real hs = Real(0.5 * kEta * c->omega);
    const double kn = Reflect ? double(c->restart_iter + step + 2) : 1.0;
    const Real lwn = Real(kn / (kn + 1.0)), rwn = Real(1.0 / (kn + 1.0));
    int2 ij[EPT];
    Real sw[EPT], u1[EPT], u0[EPT];
    int at1[EPT];   // where slot 1 goes: the edge (pull) or its second-end position (push)
#pragma unroll
    for (int t = 0; t < EPT; ++t) {
        const int e = base + t * kBlock;
        if (e < d.m) {
            ij[t] = d.ends[e];
            sw[t] = d.w[e];
            u1[t] = Reflect ? d.pred[e] : ysrc[e];
            u0[t] = Reflect ? d.u0[e] : u1[t];
            at1[t] = Pull ? e : d.colpos[e];
        }
    }
    Real ri[EPT], rj[EPT];
#pragma unroll
    for (int t = 0; t < EPT; ++t) {
        if (base + t * kBlock < d.m) {
            const bool ok = index_ok(unsigned(ij[t].x) < unsigned(d.n) && unsigned(ij[t].y) < unsigned(d.n),
                                     &d.ctl->status);
            ri[t] = ok ? d.r[ij[t].x] : Real(0);
            rj[t] = ok ? d.r[ij[t].y] : Real(0);
            if (!ok) ij[t] = make_int2(0, 0);   // the check's gathers below stay in range
        }
    }
    double acc[kEdgeSums] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int t = 0; t < EPT; ++t) {
        const int e = base + t * kBlock;
        if (e >= d.m) continue;
        const bool cov = sw[t] > Real(0);
        const Real w = cov ? sw[t] : -sw[t];
        const Real u2 = cov ? clampv(rfma(hs, (Real(1) - ri[t]) - rj[t], u1[t]), -w, Real(0))
                            : clampv(rfma(hs, rj[t] - ri[t], u1[t]), Real(0), w);
        const Real nx = rfma(lwn, rfma(Real(2), u2, -u1[t]), rmul(rwn, u0[t]));
        d.pred[e] = nx;
        const bool oka = index_ok(unsigned(at1[t]) < unsigned(d.m), &d.ctl->status);
        if (oka) d.pred1[at1[t]] = cov ? nx : w - nx;
        if (!Reflect) d.u0[e] = u1[t];
        if (Check) {
            if (Reflect) {
                d.u2s[e] = u2;
                if (oka) d.u2s1[at1[t]] = cov ? u2 : w - u2;
            }
            const double x1i = d.x1[ij[t].x], x2i = d.x2[ij[t].x];
            const double x1j = d.x1[ij[t].y], x2j = d.x2[ij[t].y];
            const double dy = double(u1[t]) - double(u2);
            const double dxi = x1i - x2i, dxj = x1j - x2j;
            acc[0] += rmul(rmul(2.0, dy), dy);
            acc[1] += rmul(cov ? dxi + dxj : dxi - dxj, dy);
            const double dr = double(u1[t]) - double(u0[t]);
            acc[2] += rmul(rmul(2.0, dr), dr);
            const double bi = bounds_at_1 ? x1i : x2i, bj = bounds_at_1 ? x1j : x2j;
            const double wd = double(w);
            acc[3] += cov ? rmul(wd, fmax(bi + bj - 1.0, 0.0)) : -rmul(wd, fmin(bi, bj));
            acc[4] += cov ? double(bounds_at_1 ? u1[t] : u2) : 0.0;
        }
    }
    if (Check) {
        block_sums<kEdgeSums>(acc, scratch, acc);
        if (threadIdx.x == 0) {
            for (int k = 0; k < kEdgeSums; ++k) d.pedge[size_t(tile) * kEdgeSums + k] = acc[k];
        }
    }
}

template <class Real, bool Reflect, bool Check, bool Pull = false>
__global__ void __launch_bounds__(kBlock)
edge_kernel(Dev<Real> d, const Real* ysrc, int step, int bounds_at_1, int gate) {
    pdl_wait();
    pdl_launch_dependents();
    edge_kernel_tile<Real, Reflect, Check, Pull>(d, blockIdx.x, ysrc, step, bounds_at_1, gate);
}

// The reflected step without check sums, on its own grid (tiles of kBlock *
// plain_edges_per_thread<Real, Pull>() edges).
template <class Real, bool Pull = false>
__global__ void __launch_bounds__(kBlock)
edge_plain_kernel(Dev<Real> d, const Real* ysrc, int step, int bounds_at_1, int gate) {
    pdl_wait();
    pdl_launch_dependents();
    edge_kernel_tile<Real, true, false, Pull, plain_edges_per_thread<Real, Pull>()>(d, blockIdx.x, ysrc, step, bounds_at_1, gate);
}

// The node part of the lower bound, sum_i min(d_i - (S^T y)_i, 0), at the
// dual (ys, yc) (solver.py:333-337), in FP64.
template <class Real, bool Wide = false, bool Pull = false>
__device__ __forceinline__ void lower_kernel_tile(const Dev<Real>& d, int tile, const Real* ys, const Real* yc) {
    if (d.ctl->terminated) return;
    __shared__ double scratch[32];
    Real* stage = warp_stage<Real, stage_runs<Wide>()>();
    const int lane = threadIdx.x & 31;
    const long long base = (long long)tile * blockDim.x + (threadIdx.x & ~31);
    const long long i = base + lane;
    const double s = scatter_at<Real, double, Wide, Pull>(d, ys, yc, base, lane, stage);
    double acc[1] = {0.0};
    if (i < d.n) {
        const double rc = double(d.diag[i]) - s;
        acc[0] = rc < 0.0 ? rc : 0.0;
    }
    block_sums<1>(acc, scratch, acc);
    if (threadIdx.x == 0) d.plower[tile] = acc[0];
}

template <class Real, bool Wide = false, bool Pull = false>
__global__ void __launch_bounds__(kBlock)
lower_kernel(Dev<Real> d, const Real* __restrict__ ys, const Real* __restrict__ yc) {
    pdl_wait();
    pdl_launch_dependents();
    lower_kernel_tile<Real, Wide, Pull>(d, blockIdx.x, ys, yc);
}

__device__ __forceinline__ double canonical(const double* node, const double* edge, double omega) {
    // + cross term (halpern_operator.py:7-35)
    const double v = (omega / kEta) * node[0] + (1.0 / (kEta * omega)) * edge[0] + 2.0 * edge[1];
    return sqrt(v > 0.0 ? v : 0.0);
}

__device__ __forceinline__ bool should_stop(double gap, long long iteration, const Params& p) {
    const bool within = iteration < p.max_iter || p.max_iter < 0;
    const bool outside = !(gap <= p.tolerance);   // NaN keeps going
    return !(within && outside);
}

// mode 0: the check before the loop (bounds at (x1, y1));
// mode 1: the check after an op_steps block (solver.py:397-469);
// mode 2: after the restart step, the new fixed-point error.
__device__ __forceinline__ void check_body(Control* c, Params p, const double* scale_ptr, const double* pnode,
                                           int nbn, const double* pedge, int nbe, const double* plower, int nbl,
                                           int mode) {
    if (c->terminated) return;
    if (mode == 2 && !c->restart) return;
    __shared__ double scratch[kEdgeSums * 32];
    __shared__ double node[kNodeSums], edge[kEdgeSums], low[1];
    reduce_rows<kNodeSums>(pnode, nbn, scratch, node);
    reduce_rows<kEdgeSums>(pedge, nbe, scratch, edge);
    if (mode != 2) reduce_rows<1>(plower, nbl, scratch, low);
    if (threadIdx.x != 0) return;
    if (mode == 2) {
        c->fp_error = canonical(node, edge, c->omega);
        c->check_error = INFINITY;
        c->restart_iter = 0;
        c->restart = 0;
        return;
    }
    const double scale = *scale_ptr;
    const double upper = (node[2] + edge[3]) * scale;
    const double lower = (low[0] + edge[4]) * scale;
    const double gap = (upper - lower) / (1.0 + fabs(upper) + fabs(lower));
    c->upper = upper;
    c->lower = lower;
    c->gap = gap;
    if (mode == 0) {
        c->fp_error = canonical(node, edge, c->omega);
        c->new_error = c->fp_error;
        c->check_error = INFINITY;
        c->terminated = should_stop(gap, c->iteration, p) ? 1 : 0;
        c->result_slot = 1;
        c->restart = 0;
        trace_put(p.trace, p.trace_cap, c->trace_len, c->iteration, gap, c->fp_error, c->omega, lower, upper, -1,
                  c->terminated);
        return;
    }
    c->iteration += p.op_steps;
    c->restart_iter += p.op_steps;
    const double new_err = canonical(node, edge, c->omega);
    c->new_error = new_err;
    const bool terminated = should_stop(gap, c->iteration, p);
    const bool sufficient = new_err <= p.beta_sufficient * c->fp_error;
    const bool necessary = new_err <= p.beta_necessary * c->fp_error && new_err > c->check_error;
    const bool artificial = double(c->restart_iter) >= p.beta_artificial * double(c->iteration);
    const bool restart = sufficient || necessary || artificial;
    if (restart) {
        const double pn = sqrt(node[1]), dn = sqrt(edge[2]);
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
    } else if (restart) {
        c->restart = 1;
    } else {
        c->check_error = new_err;
    }
    const int kind = (terminated || !restart) ? 0 : (sufficient ? 1 : (necessary ? 2 : 3));
    trace_put(p.trace, p.trace_cap, c->trace_len, c->iteration, gap, new_err, c->omega, lower, upper, kind,
              terminated ? 1 : 0);
}

__global__ void __launch_bounds__(kCheckBlock)
check_kernel(Control* c, Params p, const double* __restrict__ scale_ptr,
             const double* __restrict__ pnode, int nbn, const double* __restrict__ pedge, int nbe,
             const double* __restrict__ plower, int nbl, int mode) {
    pdl_wait();
    pdl_launch_dependents();
    check_body(c, p, scale_ptr, pnode, nbn, pedge, nbe, plower, nbl, mode);
}

// The head of a captured check block: the block's body runs only while the
// solve has not terminated (a block queued behind the one that ended the
// solve then costs this one launch instead of its ~37 gated kernels).
__global__ void block_gate_kernel(const Control* c, cudaGraphConditionalHandle body) {
    if (threadIdx.x == 0) cudaGraphSetConditional(body, c->terminated ? 0u : 1u);
}

// ---- the persistent kernel for small instances ----------------------------
// One cooperative launch runs a whole check block: op_steps steps of the node
// half and the edge half, the lower-bound pass, the check and the gated
// restart step -- the graph's tile functions in the graph's order with the
// graph's CTA shape, so the results are the graph's bit for bit -- each
// phase's tiles dealt round-robin to the resident CTAs and the phases
// separated by grid barriers (bounded waits, common.cuh; a grid of one CTA,
// as for a few hundred nodes, needs only block barriers).  For instances of a
// few thousand edges a kernel boundary costs more than the phase it ends.  The
// tile functions take the iterates through plain pointers (no __restrict__):
// here a buffer one phase reads, another phase of the same launch writes.  A
// barrier that runs out sets Control::status to kMegaWaitStatus.
constexpr int kMegaWaitStatus = 1;

struct MegaArgs {
    GridBar* bar;
    unsigned expect;                 // CTAs each barrier waits for (the grid)
    unsigned long long wait_ns;      // a barrier's wait limit
    int nb_node, nb_edge;            // tiles of the node and edge halves
};

template <class Real, bool Reflect, bool Check, bool Wide>
__device__ __forceinline__ void mega_node(const Dev<Real>& d, const MegaArgs& a, const Real* ys, const Real* yc,
                                          int step, int gate, int bounds_at_1 = 0) {
    for (int t = int(blockIdx.x); t < a.nb_node; t += gridDim.x) {
        node_kernel_tile<Real, Reflect, Check, Wide, false>(d, t, ys, yc, step, bounds_at_1, gate);
        __syncthreads();   // the next tile reuses the staging buffer
    }
}

template <class Real, bool Reflect, bool Check>
__device__ __forceinline__ void mega_edge(const Dev<Real>& d, const MegaArgs& a, const Real* ysrc, int step,
                                          int gate, int bounds_at_1 = 0) {
    for (int t = int(blockIdx.x); t < a.nb_edge; t += gridDim.x) {
        edge_kernel_tile<Real, Reflect, Check, false>(d, t, ysrc, step, bounds_at_1, gate);
        __syncthreads();
    }
}

template <class Real, bool Wide>
__device__ __forceinline__ void mega_lower(const Dev<Real>& d, const MegaArgs& a, const Real* ys, const Real* yc) {
    for (int t = int(blockIdx.x); t < a.nb_node; t += gridDim.x) {
        lower_kernel_tile<Real, Wide, false>(d, t, ys, yc);
        __syncthreads();
    }
}

// One check block (enqueue_steps' kernels, in their order); false when a
// barrier ran out.  `sync` is the barrier between phases.
template <class Real, bool Wide, class Sync>
__device__ __forceinline__ bool mega_block_body(const Dev<Real>& d, const Params& prm, const MegaArgs& a,
                                                Sync& sync) {
    const int op = int(prm.op_steps);
    for (int s = 0; s < op; ++s) {
        if (s + 1 < op)
            mega_node<Real, true, false, Wide>(d, a, d.pred, d.pred1, s, 0);
        else
            mega_node<Real, true, true, Wide>(d, a, d.pred, d.pred1, s, 0);
        if (!sync()) return false;
        if (d.m) {
            if (s + 1 < op)
                mega_edge<Real, true, false>(d, a, nullptr, s, 0);
            else
                mega_edge<Real, true, true>(d, a, nullptr, s, 0);
            if (!sync()) return false;
        }
    }
    mega_lower<Real, Wide>(d, a, d.u2s, d.u2s1);
    if (!sync()) return false;
    if (blockIdx.x == 0)
        check_body(d.ctl, prm, d.scale, d.pnode, a.nb_node, d.pedge, a.nb_edge, d.plower, a.nb_node, 1);
    if (!sync()) return false;
    if (!d.ctl->restart) return true;   // uniform: the check above is the last writer
    mega_node<Real, false, true, Wide>(d, a, d.u2s, d.u2s1, 0, 1);
    if (!sync()) return false;
    if (d.m) {
        mega_edge<Real, false, true>(d, a, d.u2s, 0, 1);
        if (!sync()) return false;
    }
    if (blockIdx.x == 0)
        check_body(d.ctl, prm, d.scale, d.pnode, a.nb_node, d.pedge, a.nb_edge, d.plower, a.nb_node, 2);
    return true;
}

// CTAs of kBlock threads of `fn` the current device holds at once.
template <class Fn>
cudaError_t grid_capacity(Fn fn, int* out) {
    int dev = 0, sms = 0, per_sm = 0;
    RB_CUDA_TRY(cudaGetDevice(&dev));
    RB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    RB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, 0));
    *out = sms * per_sm;
    return cudaSuccess;
}

// The push layout only (the slot-1 pull layout is for edge arrays beyond L2).
template <class Real, bool Wide>
__global__ void __launch_bounds__(kBlock, 1)
mega_block_kernel(const __grid_constant__ Dev<Real> d, const __grid_constant__ Params prm, MegaArgs a) {
    auto sync = [&]() {
        if (grid_sync(a.bar, a.expect, a.wait_ns)) return true;
        if (threadIdx.x == 0) d.ctl->status = kMegaWaitStatus;
        return false;
    };
    mega_block_body<Real, Wide>(d, prm, a, sync);
}

// ---- the whole solve in one CTA's shared memory (a few thousand edges) ----
// For a few hundred nodes the per-kernel graph and the grid form both wait on
// latency: the generic tiles stage every gather through L2 in 256-thread
// CTAs.  tiny_solve_kernel copies the instance into one 1024-thread CTA's
// shared memory and runs the start step, the check before the loop and up to
// `max_blocks` check blocks there, with block barriers between phases, then
// copies the iterates and the control block back.  It keeps the graph's
// arithmetic term for term, so its results are the graph's bit for bit:
// * a node's S^T y is its first-end run, then its second-end run, each added
//   in order from zero (warp_runs' sums), one thread per node;
// * edge tiles keep their shape: thread t of the block's half q works tile
//   q (+2, +4, ...) as thread t of a 256-thread CTA would, kEdgesPerThread
//   edges a kBlock apart, in order;
// * per-tile check sums are block_sums over the half (butterfly in each
//   warp, then the half's first warp adds its 8 warp totals in order), and
//   check_body's row reductions see at most 256 rows, which 512 threads add
//   in the order 256 threads do.
constexpr int kTinyThreads = 512;   // 128 registers a thread (1024 threads spill)
constexpr int kTinyParts = kTinyThreads / kBlock;

struct TinyLayout {
    size_t x1, x2, x0, r, diag, deg, row_ptr, col_ptr, ends, w, colpos, pred, pred1, u0, u2s, u2s1;
    size_t pnode, pedge, plower, ctl, scale, total;
};

__host__ __device__ inline size_t tiny_take(size_t& at, size_t bytes) {
    const size_t here = at;
    at = (at + bytes + 15) & ~size_t(15);
    return here;
}

__host__ __device__ inline TinyLayout tiny_layout(long long n, long long m, int nb_node, int nb_edge, int real) {
    TinyLayout t{};
    size_t at = 0;
    t.x1 = tiny_take(at, size_t(n) * real);
    t.x2 = tiny_take(at, size_t(n) * real);
    t.x0 = tiny_take(at, size_t(n) * real);
    t.r = tiny_take(at, size_t(n) * real);
    t.diag = tiny_take(at, size_t(n) * real);
    t.deg = tiny_take(at, size_t(n) * real);
    t.row_ptr = tiny_take(at, size_t(n + 1) * sizeof(int));
    t.col_ptr = tiny_take(at, size_t(n + 1) * sizeof(int));
    t.ends = tiny_take(at, size_t(m) * sizeof(int2));
    t.w = tiny_take(at, size_t(m) * real);
    t.colpos = tiny_take(at, size_t(m) * sizeof(int));
    t.pred = tiny_take(at, size_t(m) * real);
    t.pred1 = tiny_take(at, size_t(m) * real);
    t.u0 = tiny_take(at, size_t(m) * real);
    t.u2s = tiny_take(at, size_t(m) * real);
    t.u2s1 = tiny_take(at, size_t(m) * real);
    t.pnode = tiny_take(at, size_t(nb_node) * kNodeSums * sizeof(double));
    t.pedge = tiny_take(at, size_t(nb_edge) * kEdgeSums * sizeof(double));
    t.plower = tiny_take(at, size_t(nb_node) * sizeof(double));
    t.ctl = tiny_take(at, sizeof(Control));
    t.scale = tiny_take(at, sizeof(double));
    t.total = at;
    return t;
}

template <class T>
__device__ __forceinline__ void tiny_copy(T* dst, const T* src, long long count) {
    for (long long i = threadIdx.x; i < count; i += blockDim.x) dst[i] = src[i];
}

// block_sums over this thread's 256-thread part of the block: the part's totals
// land in out[q * K + k].  Every thread of the block calls it.
template <int K>
__device__ __forceinline__ void part_sums(const double (&v)[K], double* scratch, double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = warp >> 3, wq = warp & 7;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const double s = warp_sum(v[k]);
        if (lane == 0) scratch[(q * K + k) * 32 + wq] = s;
    }
    __syncthreads();
    if (wq == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = lane < kBlock / 32 ? scratch[(q * K + k) * 32 + lane] : 0.0;
            s = warp_sum(s);
            if (lane == 0) out[q * K + k] = s;
        }
    }
    __syncthreads();
}

// A run of `v` added in order from zero.
template <class Acc, class Real>
__device__ __forceinline__ Acc tiny_run(const int* ptr, const Real* v, int i, int m, int* status) {
    Acc s = Acc(0);
    const int k0 = ptr[i], e = ptr[i + 1];
    if (!index_ok(0 <= k0 && k0 <= e && e <= m, status)) return s;
    for (int k = k0; k < e; ++k) s += Acc(v[k]);
    return s;
}

// node_kernel_tile's step, term for term, one thread per node.
template <class Real, bool Reflect, bool Check>
__device__ __forceinline__ void tiny_node(const Dev<Real>& d, const Real* ys, const Real* yc, int step, int bounds_at_1,
                                          int gate, int nb_node, double* scratch, double* qout) {
    const Control* c = d.ctl;
    if (skip(c, gate)) return;
    for (int base = 0; base < nb_node * kBlock; base += kTinyThreads) {
        const int i = base + int(threadIdx.x);
        double acc[kNodeSums] = {0.0, 0.0, 0.0};
        if (i < d.n) {
            const Real x2o = d.x2[i], di = d.diag[i], dg = d.deg[i];
            Real x1o = Real(0), x0o = Real(0);
            if (Reflect) {
                x1o = d.x1[i];
                x0o = d.x0[i];
            }
            const Real s0 = tiny_run<Real>(d.row_ptr, ys, i, d.m, &d.ctl->status);
            const Real s1 = tiny_run<Real>(d.col_ptr, yc, i, d.m, &d.ctl->status);
            const Real s = s0 + s1;
            Real x1v;
            if (Reflect) {
                const double k = double(c->restart_iter + step + 1);
                const Real lw = Real(k / (k + 1.0)), rw = Real(1.0 / (k + 1.0));
                x1v = rfma(lw, rfma(Real(2), x2o, -x1o), rmul(rw, x0o));
            } else {
                x1v = x2o;
            }
            const Real ps = Real(kEta / c->omega);
            const Real x2v = clampv(rfma(-ps, (di - s) / dg, x1v), Real(0), Real(1));
            d.x1[i] = x1v;
            d.x2[i] = x2v;
            d.r[i] = rfma(Real(2), x2v, -x1v);
            if (!Reflect) d.x0[i] = x1v;
            if (Check) {
                const double dx = double(x1v) - double(x2v);
                const double dr = Reflect ? double(x1v) - double(x0o) : 0.0;
                acc[0] = double(dg) * dx * dx;
                acc[1] = double(dg) * dr * dr;
                acc[2] = double(di) * double(bounds_at_1 ? x1v : x2v);
            }
        }
        if (Check) {
            part_sums<kNodeSums>(acc, scratch, qout);
            const int tile = base / kBlock + int(threadIdx.x >> 8);
            if ((threadIdx.x & (kBlock - 1)) == 0 && tile < nb_node)
                for (int k = 0; k < kNodeSums; ++k) d.pnode[size_t(tile) * kNodeSums + k] = qout[(threadIdx.x >> 8) * kNodeSums + k];
        }
    }
}

// edge_kernel_tile's step, term for term, the tiles two at a time.
template <class Real, bool Reflect, bool Check>
__device__ __forceinline__ void tiny_edge(const Dev<Real>& d, const Real* ysrc, int step, int bounds_at_1, int gate,
                                          int nb_edge, double* scratch, double* qout) {
    const Control* c = d.ctl;
    if (skip(c, gate)) return;
    const Real hs = Real(0.5 * kEta * c->omega);
    const double kn = Reflect ? double(c->restart_iter + step + 2) : 1.0;
    const Real lwn = Real(kn / (kn + 1.0)), rwn = Real(1.0 / (kn + 1.0));
    const int q = int(threadIdx.x >> 8), t = int(threadIdx.x & (kBlock - 1));
    for (int tile0 = 0; tile0 < nb_edge; tile0 += kTinyParts) {
        const int tile = tile0 + q;
        const int base = tile * (kBlock * kEdgesPerThread) + t;
        double acc[kEdgeSums] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int u = 0; u < kEdgesPerThread; ++u) {
            const int e = base + u * kBlock;
            if (tile >= nb_edge || e >= d.m) continue;
            const int2 ij = d.ends[e];
            const Real sw = d.w[e];
            const Real u1 = Reflect ? d.pred[e] : ysrc[e];
            const Real u0 = Reflect ? d.u0[e] : u1;
            const int at1 = d.colpos[e];
            const bool ok = index_ok(unsigned(ij.x) < unsigned(d.n) && unsigned(ij.y) < unsigned(d.n),
                                     &d.ctl->status);
            const int2 ijs = ok ? ij : make_int2(0, 0);   // every gather below stays in range
            const Real ri = d.r[ijs.x], rj = d.r[ijs.y];
            const bool cov = sw > Real(0);
            const Real w = cov ? sw : -sw;
            const Real u2 = cov ? clampv(rfma(hs, (Real(1) - ri) - rj, u1), -w, Real(0))
                                : clampv(rfma(hs, rj - ri, u1), Real(0), w);
            const Real nx = rfma(lwn, rfma(Real(2), u2, -u1), rmul(rwn, u0));
            d.pred[e] = nx;
            const bool oka = index_ok(unsigned(at1) < unsigned(d.m), &d.ctl->status);
            if (oka) d.pred1[at1] = cov ? nx : w - nx;
            if (!Reflect) d.u0[e] = u1;
            if (Check) {
                if (Reflect) {
                    d.u2s[e] = u2;
                    if (oka) d.u2s1[at1] = cov ? u2 : w - u2;
                }
                const double x1i = d.x1[ijs.x], x2i = d.x2[ijs.x];
                const double x1j = d.x1[ijs.y], x2j = d.x2[ijs.y];
                const double dy = double(u1) - double(u2);
                const double dxi = x1i - x2i, dxj = x1j - x2j;
                acc[0] += rmul(rmul(2.0, dy), dy);
                acc[1] += rmul(cov ? dxi + dxj : dxi - dxj, dy);
                const double dr = double(u1) - double(u0);
                acc[2] += rmul(rmul(2.0, dr), dr);
                const double bi = bounds_at_1 ? x1i : x2i, bj = bounds_at_1 ? x1j : x2j;
                const double wd = double(w);
                acc[3] += cov ? rmul(wd, fmax(bi + bj - 1.0, 0.0)) : -rmul(wd, fmin(bi, bj));
                acc[4] += cov ? double(bounds_at_1 ? u1 : u2) : 0.0;
            }
        }
        if (Check) {
            part_sums<kEdgeSums>(acc, scratch, qout);
            if (t == 0 && tile < nb_edge)
                for (int k = 0; k < kEdgeSums; ++k) d.pedge[size_t(tile) * kEdgeSums + k] = qout[q * kEdgeSums + k];
        }
    }
}

// lower_kernel_tile's pass, term for term, one thread per node.
template <class Real>
__device__ __forceinline__ void tiny_lower(const Dev<Real>& d, const Real* ys, const Real* yc, int nb_node,
                                           double* scratch, double* qout) {
    if (d.ctl->terminated) return;
    for (int base = 0; base < nb_node * kBlock; base += kTinyThreads) {
        const int i = base + int(threadIdx.x);
        double acc[1] = {0.0};
        if (i < d.n) {
            const double s0 = tiny_run<double>(d.row_ptr, ys, i, d.m, &d.ctl->status);
            const double s1 = tiny_run<double>(d.col_ptr, yc, i, d.m, &d.ctl->status);
            const double s = s0 + s1;
            const double rc = double(d.diag[i]) - s;
            acc[0] = rc < 0.0 ? rc : 0.0;
        }
        part_sums<1>(acc, scratch, qout);
        const int tile = base / kBlock + int(threadIdx.x >> 8);
        if ((threadIdx.x & (kBlock - 1)) == 0 && tile < nb_node) d.plower[tile] = qout[threadIdx.x >> 8];
    }
}

// check_body, out of line: its row reductions hold many values at once, and
// inlined they would hold registers through the whole step loop.
__device__ __noinline__ void tiny_check(Control* c, const Params& prm, const double* scale, const double* pnode,
                                        int nbn, const double* pedge, int nbe, const double* plower, int mode) {
    check_body(c, prm, scale, pnode, nbn, pedge, nbe, plower, nbn, mode);
}

// start: run the start step and the check before the loop first (after
// init_kernel or warm_init_kernel has set the start point in global memory).
template <class Real>
__global__ void __launch_bounds__(kTinyThreads, 1)
tiny_solve_kernel(const __grid_constant__ Dev<Real> g, const __grid_constant__ Params prm, int nb_node, int nb_edge,
                  int start, int max_blocks) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ Dev<Real> d;
    __shared__ double scratch[kTinyParts * kEdgeSums * 32];
    __shared__ double qout[kTinyParts * kEdgeSums];
    const TinyLayout L = tiny_layout(g.n, g.m, nb_node, nb_edge, int(sizeof(Real)));
    auto at = [&](size_t off) { return static_cast<void*>(smem_raw + off); };
    if (threadIdx.x == 0) {
        d = g;
        d.x1 = static_cast<Real*>(at(L.x1));
        d.x2 = static_cast<Real*>(at(L.x2));
        d.x0 = static_cast<Real*>(at(L.x0));
        d.r = static_cast<Real*>(at(L.r));
        d.diag = static_cast<const Real*>(at(L.diag));
        d.deg = static_cast<const Real*>(at(L.deg));
        d.row_ptr = static_cast<const int*>(at(L.row_ptr));
        d.col_ptr = static_cast<const int*>(at(L.col_ptr));
        d.ends = static_cast<const int2*>(at(L.ends));
        d.w = static_cast<const Real*>(at(L.w));
        d.colpos = static_cast<const int*>(at(L.colpos));
        d.pred = static_cast<Real*>(at(L.pred));
        d.pred1 = static_cast<Real*>(at(L.pred1));
        d.u0 = static_cast<Real*>(at(L.u0));
        d.u2s = static_cast<Real*>(at(L.u2s));
        d.u2s1 = static_cast<Real*>(at(L.u2s1));
        d.pnode = static_cast<double*>(at(L.pnode));
        d.pedge = static_cast<double*>(at(L.pedge));
        d.plower = static_cast<double*>(at(L.plower));
        d.ctl = static_cast<Control*>(at(L.ctl));
        d.scale = static_cast<const double*>(at(L.scale));
        *d.ctl = *g.ctl;
        *static_cast<double*>(at(L.scale)) = *g.scale;
    }
    const long long n = g.n, m = g.m;
    tiny_copy(static_cast<Real*>(at(L.x1)), g.x1, n);
    tiny_copy(static_cast<Real*>(at(L.x2)), g.x2, n);
    tiny_copy(static_cast<Real*>(at(L.x0)), g.x0, n);
    tiny_copy(static_cast<Real*>(at(L.r)), g.r, n);
    tiny_copy(static_cast<Real*>(at(L.diag)), g.diag, n);
    tiny_copy(static_cast<Real*>(at(L.deg)), g.deg, n);
    tiny_copy(static_cast<int*>(at(L.row_ptr)), g.row_ptr, n + 1);
    tiny_copy(static_cast<int*>(at(L.col_ptr)), g.col_ptr, n + 1);
    tiny_copy(static_cast<int2*>(at(L.ends)), g.ends, m);
    tiny_copy(static_cast<Real*>(at(L.w)), g.w, m);
    tiny_copy(static_cast<int*>(at(L.colpos)), g.colpos, m);
    tiny_copy(static_cast<Real*>(at(L.pred)), g.pred, m);
    tiny_copy(static_cast<Real*>(at(L.pred1)), g.pred1, m);
    tiny_copy(static_cast<Real*>(at(L.u0)), g.u0, m);
    tiny_copy(static_cast<Real*>(at(L.u2s)), g.u2s, m);
    tiny_copy(static_cast<Real*>(at(L.u2s1)), g.u2s1, m);
    // with no edges no edge tile writes its partial row, which the checks read
    for (int i = threadIdx.x; i < nb_edge * kEdgeSums; i += blockDim.x)
        static_cast<double*>(at(L.pedge))[i] = 0.0;
    __syncthreads();
    if (start) {
        // x1, y1 = _raw_step(x0, y0) with the bounds at the start point
        // (start_step's kernels), then the check before the loop
        tiny_node<Real, false, true>(d, d.pred, d.pred1, 0, 1, 0, nb_node, scratch, qout);
        tiny_lower<Real>(d, d.pred, d.pred1, nb_node, scratch, qout);
        __syncthreads();
        if (m) {
            tiny_edge<Real, false, true>(d, d.pred, 0, 1, 0, nb_edge, scratch, qout);
            __syncthreads();
        }
        tiny_check(d.ctl, prm, d.scale, d.pnode, nb_node, d.pedge, nb_edge, d.plower, 0);
        __syncthreads();
    }
    const int op = int(prm.op_steps);
    for (int b = 0; b < max_blocks && !d.ctl->terminated; ++b) {
        // one check block: enqueue_steps' kernels, in their order
        for (int s = 0; s < op; ++s) {
            if (s + 1 < op)
                tiny_node<Real, true, false>(d, d.pred, d.pred1, s, 0, 0, nb_node, scratch, qout);
            else
                tiny_node<Real, true, true>(d, d.pred, d.pred1, s, 0, 0, nb_node, scratch, qout);
            __syncthreads();
            if (m) {
                if (s + 1 < op)
                    tiny_edge<Real, true, false>(d, nullptr, s, 0, 0, nb_edge, scratch, qout);
                else
                    tiny_edge<Real, true, true>(d, nullptr, s, 0, 0, nb_edge, scratch, qout);
                __syncthreads();
            }
        }
        tiny_lower<Real>(d, d.u2s, d.u2s1, nb_node, scratch, qout);
        __syncthreads();
        tiny_check(d.ctl, prm, d.scale, d.pnode, nb_node, d.pedge, nb_edge, d.plower, 1);
        __syncthreads();
        if (d.ctl->restart) {
            tiny_node<Real, false, true>(d, d.u2s, d.u2s1, 0, 0, 1, nb_node, scratch, qout);
            __syncthreads();
            if (m) {
                tiny_edge<Real, false, true>(d, d.u2s, 0, 0, 1, nb_edge, scratch, qout);
                __syncthreads();
            }
            tiny_check(d.ctl, prm, d.scale, d.pnode, nb_node, d.pedge, nb_edge, d.plower, 2);
            __syncthreads();
        }
    }
    tiny_copy(g.x1, d.x1, n);
    tiny_copy(g.x2, d.x2, n);
    tiny_copy(g.x0, d.x0, n);
    tiny_copy(g.r, d.r, n);
    tiny_copy(g.pred, d.pred, m);
    tiny_copy(g.pred1, d.pred1, m);
    tiny_copy(g.u0, d.u0, m);
    tiny_copy(g.u2s, d.u2s, m);
    tiny_copy(g.u2s1, d.u2s1, m);
    if (threadIdx.x == 0) *g.ctl = *d.ctl;
}

// Cold start: the centroid, x = 1/2 and y_e = (-W_ij, -W_ij) / scale, which is
// u = -w / 2 in the one-coordinate form (half_edge.py:87-94).
template <class Real>
__global__ void init_kernel(Dev<Real> d, Control* c, double omega, double theta) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < d.n) {
        d.x1[k] = Real(0.5);
        d.x2[k] = Real(0.5);
        d.x0[k] = Real(0.5);
    }
    if (k < d.m) {
        const Real sw = d.w[k];
        const Real u = Real(-0.5) * sw;
        const Real v = sw > Real(0) ? u : -sw - u;
        d.u0[k] = u;
        d.pred[k] = u;
        d.u2s[k] = u;
        const long long at = d.pull ? k : d.colpos[k];
        d.pred1[at] = v;
        d.u2s1[at] = v;
    }
    if (k == 0) {
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
        c->trace_len = 0;
    }
}

// A warm start (qubo/praq-jax/praq/solver.py:482-560): the given primal
// clipped to [0, 1]^n and the given half-edge dual pairs (instance units,
// input edge order, wy[2e], wy[2e+1]) scaled and projected onto each edge's
// dual set (projection.py:16-42), in the one-coordinate form.  NULL wx keeps
// x = 1/2, NULL wy keeps the centroid.  Everything else as init_kernel.
template <class Real>
__global__ void warm_init_kernel(Dev<Real> d, Control* c, double omega, double theta,
                                 const double* __restrict__ wx, const double* __restrict__ wy,
                                 const int* __restrict__ perm) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < d.n) {
        const Real x = wx ? Real(fmin(fmax(wx[k], 0.0), 1.0)) : Real(0.5);
        d.x1[k] = x;
        d.x2[k] = x;
        d.x0[k] = x;
    }
    if (k < d.m) {
        const Real sw = d.w[k];
        Real u = Real(-0.5) * sw;
        if (wy) {
            const long long e = perm ? perm[k] : k;
            const double sc = *d.scale;
            const double v1 = wy[2 * e] / sc, v2 = wy[2 * e + 1] / sc, swd = double(sw);
            u = swd > 0.0 ? Real(fmin(fmax(0.5 * (v1 + v2), -swd), 0.0))                  // covering
                           : Real(fmin(fmax(v1 + 0.5 * (-swd - v1 - v2), 0.0), -swd));   // packing
        }
        const Real v = sw > Real(0) ? u : -sw - u;
        d.u0[k] = u;
        d.pred[k] = u;
        d.u2s[k] = u;
        const long long at = d.pull ? k : d.colpos[k];
        d.pred1[at] = v;
        d.u2s1[at] = v;
    }
    if (k == 0) {
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
        c->trace_len = 0;
    }
}

// ---------------------------------------------------------------------------
// device preprocessing (the reference does this on the host:
// qubo/praq-cuda/src/solver.cuh:517-569 and qubo/praq-cuda/src/praq.cu:35-79)

// Per edge: range and self-loop check (bit 0 of *flags), first-end order check
// (bit 1 when some first end is smaller than its predecessor's), int32 keys,
// and the squares of the objective vector (fixed grid, fixed order).
__global__ void prep_scan_kernel(long long n, long long m, const int64_t* __restrict__ rows,
                                 const int64_t* __restrict__ cols, const double* __restrict__ vals,
                                 const double* __restrict__ diag, int* __restrict__ krow,
                                 int* __restrict__ kcol, int* flags, double* __restrict__ partial) {
    __shared__ double scratch[32];
    double sq = 0.0;
    int bad = 0, unsorted = 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
        const int64_t i = rows[e], j = cols[e];
        if (i < 0 || i >= n || j < 0 || j >= n || i == j) bad = 1;
        if (e > 0 && rows[e - 1] > i) unsorted = 1;
        krow[e] = int(i);
        kcol[e] = int(j);
        const double v = vals[e];
        sq += 4.0 * v * v;
    }
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double v = diag[i];
        sq += v * v;
    }
    if (bad) atomicOr(flags, 1);
    if (unsorted) atomicOr(flags, 2);
    double acc[1] = {sq};
    block_sums<1>(acc, scratch, acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
}

__global__ void prep_scale_kernel(const double* __restrict__ partial, int count, double* scale) {
    __shared__ double scratch[32];
    __shared__ double total[1];
    reduce_rows<1>(partial, count, scratch, total);
    if (threadIdx.x == 0) *scale = total[0] > 0.0 ? sqrt(total[0]) : 1.0;
}

__global__ void iota_kernel(int m, int* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) out[k] = k;
}

// Sorted edge s takes input edge perm[s] (perm null: identity).
template <class Real>
__global__ void prep_edges_kernel(int m, const int* __restrict__ perm, const int* __restrict__ krow,
                                  const int* __restrict__ kcol, const double* __restrict__ vals,
                                  const double* __restrict__ scale, int2* __restrict__ ends,
                                  Real* __restrict__ w, int* __restrict__ first,
                                  int* __restrict__ second, int* __restrict__ sidx) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= m) return;
    const int e = perm ? perm[s] : s;
    const int i = krow[e], j = kcol[e];
    ends[s] = make_int2(i, j);
    w[s] = Real(2.0 * vals[e] / *scale);
    first[s] = i;
    second[s] = j;
    sidx[s] = s;
}

// ptr[v] = the first position p of the sorted `keys` with keys[p] >= v, v <= n.
__global__ void prep_runs_kernel(long long n, int m, const int* __restrict__ keys, int* __restrict__ ptr) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;   // v = n is valid: n <= INT_MAX
    if (v > n) return;
    int lo = 0, hi = m;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (keys[mid] < v) lo = mid + 1; else hi = mid;
    }
    ptr[v] = lo;
}

__global__ void prep_colpos_kernel(int m, const int* __restrict__ order, int* __restrict__ colpos) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) colpos[order[k]] = k;
}

template <class Real>
__global__ void prep_nodes_kernel(int n, const int* __restrict__ row_ptr, const int* __restrict__ col_ptr,
                                  const double* __restrict__ diag, const double* __restrict__ scale,
                                  Real* __restrict__ dn, Real* __restrict__ deg) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int incident = (row_ptr[i + 1] - row_ptr[i]) + (col_ptr[i + 1] - col_ptr[i]);
    deg[i] = Real(incident > 0 ? incident : 1);
    dn[i] = Real(diag[i] / *scale);
}

struct SolverBase {
    virtual ~SolverBase() = default;
    virtual int run() = 0;
    virtual int set_warm(const double* x, const double* y2) = 0;
    virtual int result(double* x, double* y2, PraqResult* r) = 0;
    virtual long long launches() const = 0;
    virtual int run_profiled(double* ms, long long* count) = 0;
    // -1 auto, 0 the graph, 1 the persistent kernel where the instance allows
    // it; *active: which one later runs take
    virtual int set_megakernel(int mode, int* active) = 0;
    virtual int set_trace(int capacity) = 0;
    virtual int get_trace(reform_trace_record* out, int capacity, int64_t* total) = 0;
    double time_limit = -1.0;   // seconds of wall clock per run; < 0: none
};

template <class Real>
struct Solver final : SolverBase {
    int n = 0, m = 0;
    Params prm{};
    PraqParameters p{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int stream_dev = -1;   // the device of an owned stream (from the library's stream pool)
    PoolBuf<int> row_ptr, col_ptr, colidx, colpos, perm;
    PoolBuf<int2> ends;
    PoolBuf<Real> w, diag, deg, x1, x2, x0, r, pred, pred1, u0, u2s, u2s1;
    PoolBuf<double> pnode, pedge, plower, scale;
    PoolBuf<double> warm_x, warm_y;   // a warm start (instance units), optional
    PoolBuf<Control> ctl;
    Control* mirror = nullptr;   // pinned host copy of the control block
    Dev<Real> d{};
    int nb_node = 1, nb_edge = 1, nb_edge_push = 1, nb_edge_pull = 1;
    bool wide = false;   // node gather of both runs at once (warp_runs2)
    bool pull = false;   // slot-1 layout (see the layout notes at the top)
    bool allow_pull = true;   // false: always push (the batched engine's kernels)
    bool allow_mega = true;   // false: never the persistent kernel (the batched engine's instances)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t done[2] = {nullptr, nullptr};
    long long nlaunch = 0, block_nodes = 0;
    bool gated = false;   // the captured block is the conditional (gated) graph
    int status_override = -100;
    int runs = 0;
    // The persistent kernel in place of the graph, in its grid form
    // (mega_block_kernel, mega_grid resident CTAs) or its single-CTA form
    // (tiny_solve_kernel): chosen at set-up or by set_mega.
    bool mega = false;
    int mega_mode = -1;              // -1 auto, 0 off, 1 on where the instance allows it
    int mega_grid = 0;
    unsigned mega_phantom = 0;       // CTAs the barriers also wait for, never launched (fault injection)
    unsigned long long mega_wait_ns = 1000000000ull;
    PoolBuf<GridBar> bar;
    PoolBuf<reform_trace_record> trace;   // the convergence-trace ring, optional
    // The whole solve in one CTA's shared memory (tiny_solve_kernel), when the
    // instance fits: tiny_smem bytes; up to kTinyBlocks check blocks a launch.
    bool tiny = false, tiny_fits = false;
    size_t tiny_smem = 0;
    static constexpr int kTinyBlocks = 128;

    ~Solver() override {
        if (stream) cudaStreamSynchronize(stream);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto& ev : done) if (ev) cudaEventDestroy(ev);
        for (auto& ev : evpool) cudaEventDestroy(ev);
        row_ptr.release(); col_ptr.release(); colidx.release(); colpos.release(); perm.release();
        ends.release();
        w.release(); diag.release(); deg.release();
        x1.release(); x2.release(); x0.release(); r.release(); pred.release(); pred1.release();
        u0.release(); u2s.release(); u2s1.release();
        pnode.release(); pedge.release(); plower.release(); scale.release(); ctl.release(); bar.release();
        trace.release();
        warm_x.release(); warm_y.release();
        if (stream) cudaStreamSynchronize(stream);
        pinned_put(mirror);
        if (own_stream && stream) stream_put(stream, stream_dev);
    }

    // Lay the instance out on the device.  Returns 0, PRAQ_ERROR_INSTANCE or
    // PRAQ_ERROR_CUDA.
    int setup(const PraqInstance& in, cudaStream_t s) {
        if (s) {
            stream = s;
        } else {
            if (stream_get(&stream, &stream_dev) != cudaSuccess) return PRAQ_ERROR_CUDA;
            own_stream = true;
        }
        mirror = static_cast<Control*>(pinned_get());
        if (!mirror) return PRAQ_ERROR_CUDA;
        std::memset(static_cast<void*>(mirror), 0, sizeof(Control));   // no run yet: no trace, nothing done
        pull = choose_pull(in.m);
        const int st = layout(in);
        if (st) return st;
        nb_node = ceil_div(n, kBlock);   // one node per thread
        nb_edge = std::max(1, ceil_div(m, kBlock * kEdgesPerThread));
        nb_edge_push = std::max(1, ceil_div(m, kBlock * plain_edges_per_thread<Real, false>()));
        nb_edge_pull = std::max(1, ceil_div(m, kBlock * plain_edges_per_thread<Real, true>()));
        // The wide gather halves a warp's chain of dependent loads but takes
        // twice the registers: it wins while the node grid is one wave of it.
        {
            int waves = 0;   // CTAs of the wide node kernel one wave holds
            const cudaError_t st = once_per_device(&waves, [](int* v) {
                int dev = 0, sms = 0, per_sm = 0;
                RB_CUDA_TRY(cudaGetDevice(&dev));
                RB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
                RB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, node_kernel<Real, true, false, true>,
                                                                          kBlock, 0));
                *v = sms * per_sm;
                return cudaSuccess;
            });
            if (st != cudaSuccess) return PRAQ_ERROR_CUDA;
            wide = kGather == 1 || (kGather == 2 && nb_node <= waves);
        }
        for (auto* b : {&x1, &x2, &x0, &r})
            if (b->alloc(n, stream)) return PRAQ_ERROR_CUDA;
        for (auto* b : {&pred, &pred1, &u0, &u2s, &u2s1})
            if (b->alloc(m, stream)) return PRAQ_ERROR_CUDA;
        if (pnode.alloc(size_t(nb_node) * kNodeSums, stream) ||
            pedge.alloc(size_t(nb_edge) * kEdgeSums, stream) || plower.alloc(nb_node, stream) ||
            ctl.alloc(1, stream))
            return PRAQ_ERROR_CUDA;
        // With no edges no edge kernel ever writes its partial row, which the
        // checks still read: it must hold zeros, not what the pool last held.
        if (cudaMemsetAsync(pedge.ptr, 0, sizeof(double) * pedge.count, stream) ||
            cudaMemsetAsync(pnode.ptr, 0, sizeof(double) * pnode.count, stream) ||
            cudaMemsetAsync(plower.ptr, 0, sizeof(double) * plower.count, stream))
            return PRAQ_ERROR_CUDA;
        for (auto& ev : done)
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return PRAQ_ERROR_CUDA;
        d.n = n; d.m = m;
        d.row_ptr = row_ptr.ptr; d.col_ptr = col_ptr.ptr;
        d.pull = pull ? 1 : 0;
        d.colidx = pull ? colidx.ptr : nullptr;
        d.colpos = pull ? nullptr : colpos.ptr;
        d.ends = ends.ptr; d.w = w.ptr; d.diag = diag.ptr; d.deg = deg.ptr; d.scale = scale.ptr;
        d.x1 = x1.ptr; d.x2 = x2.ptr; d.x0 = x0.ptr; d.r = r.ptr;
        d.pred = pred.ptr; d.pred1 = pred1.ptr; d.u0 = u0.ptr; d.u2s = u2s.ptr; d.u2s1 = u2s1.ptr;
        d.pnode = pnode.ptr; d.pedge = pedge.ptr; d.plower = plower.ptr; d.ctl = ctl.ptr;
        prm.tolerance = p.tolerance;
        prm.max_iter = p.max_iter;
        prm.op_steps = p.op_steps;
        prm.beta_sufficient = p.beta_sufficient;
        prm.beta_necessary = p.beta_necessary;
        prm.beta_artificial = p.beta_artificial;
        prm.theta_target = p.theta_target;
        prm.theta_decay = p.theta_decay;
        block_nodes = (m ? 2 : 1) * (long long)p.op_steps + 2 + (m ? 2 : 1) + 1;
        if (init_mega() != cudaSuccess) return PRAQ_ERROR_CUDA;
        return cudaGetLastError() == cudaSuccess ? 0 : PRAQ_ERROR_CUDA;
    }

    // --- the persistent kernel -------------------------------------------
    cudaError_t init_mega() {
        mega_grid = 0;
        if (!allow_mega) return cudaSuccess;
        if (!pull) {
            // resident CTAs of each grid form, once per process and device
            // (one lambda per kernel: the lambda's type keys the memo)
            int cap = 0;
            if (wide) {
                RB_CUDA_TRY(once_per_device(&cap, [](int* v) { return grid_capacity(mega_block_kernel<Real, true>, v); }));
            } else {
                RB_CUDA_TRY(once_per_device(&cap, [](int* v) { return grid_capacity(mega_block_kernel<Real, false>, v); }));
            }
            // no phase has more tiles than this: more CTAs would only wait
            mega_grid = int(std::min<long long>(cap, std::max(nb_node, m ? nb_edge : 1)));
            // the single-CTA form: the instance in the shared memory its
            // static arrays leave (the kernel's limit raised to it once)
            int room = 0;
            RB_CUDA_TRY(once_per_device(&room, [](int* v) {
                int dev = 0, optin = 0;
                cudaFuncAttributes fa{};
                RB_CUDA_TRY(cudaGetDevice(&dev));
                RB_CUDA_TRY(cudaFuncGetAttributes(&fa, tiny_solve_kernel<Real>));
                RB_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
                *v = optin > int(fa.sharedSizeBytes) ? optin - int(fa.sharedSizeBytes) : 0;
                return cudaFuncSetAttribute(tiny_solve_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, *v);
            }));
            tiny_smem = tiny_layout(n, m, nb_node, nb_edge, int(sizeof(Real))).total;
            // check_body's row reductions keep the 256-thread order up to 256 rows
            tiny_fits = tiny_smem <= size_t(room) && nb_node <= kBlock && nb_edge <= kBlock;
        }
        // REFORM_PRAQ_MEGA=0|1 sets the initial mode (tests, measurements);
        // REFORM_PRAQ_MEGA_PHANTOM=k makes every barrier wait for k CTAs that
        // are never launched, so each wait runs out (the fault-injection test)
        const char* env = std::getenv("REFORM_PRAQ_MEGA");
        int mode = -1;
        if (env && (env[0] == '0' || env[0] == '1') && env[1] == '\0') mode = env[0] - '0';
        const char* ph = std::getenv("REFORM_PRAQ_MEGA_PHANTOM");
        if (ph) {
            mega_phantom = unsigned(std::strtoul(ph, nullptr, 10));
            if (mega_phantom) mega_wait_ns = 50000000ull;   // 50 ms: the test waits for every barrier
        }
        return set_mega(mode);
    }

    // mode -1: automatic (the single-CTA form for at most kTinyAutoTiles edge
    // tiles, else the graph: measured per solve, the single-CTA form is 2x
    // faster than the graph at n = 200-400 and 1.5x at n = 700, m = 2,000,
    // but 4 % slower at n = 1,500, m = 4,500; the grid form was slower than the
    // graph from n = 400 up); 0: the graph; 1: the single-CTA form when it
    // fits, else the grid form; 2: the grid form.
    static constexpr int kTinyAutoTiles = 2;
    cudaError_t set_mega(int mode) {
        mega_mode = mode < 0 ? -1 : (mode > 2 ? 2 : mode);
        tiny = tiny_fits && (mega_mode == 1 || (mega_mode == -1 && nb_edge <= kTinyAutoTiles));
        mega = !tiny && mega_mode >= 1 && mega_grid > 0;
        if (mega && !bar.ptr) {
            RB_CUDA_TRY(bar.alloc(1, stream));
            RB_CUDA_TRY(cudaMemsetAsync(bar.ptr, 0, sizeof(GridBar), stream));
        }
        return cudaSuccess;
    }

    int set_megakernel(int mode, int* active) override {
        const cudaError_t st = set_mega(mode);
        if (active) *active = tiny ? 2 : (mega ? 1 : 0);
        return st == cudaSuccess ? 0 : PRAQ_ERROR_CUDA;
    }

    cudaError_t launch_tiny(int start) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(1);
        cfg.blockDim = dim3(unsigned(kTinyThreads));
        cfg.dynamicSmemBytes = tiny_smem;
        cfg.stream = stream;
        return cudaLaunchKernelEx(&cfg, tiny_solve_kernel<Real>, d, prm, nb_node, nb_edge, start, kTinyBlocks);
    }

    // A solve in the single-CTA form: the start point set in global memory,
    // then launches of up to kTinyBlocks check blocks (the first with the
    // start step and its check) until the solve ends; the wall-clock budget
    // is checked between launches.
    int run_tiny(std::chrono::steady_clock::time_point started) {
        nlaunch = 0;
        const int count = std::max(n, m);
        if (warm_x.ptr || warm_y.ptr)
            warm_init_kernel<Real><<<ceil_div(count, kBlock), kBlock, 0, stream>>>(
                d, d.ctl, p.omega, p.theta_initial, warm_x.ptr, warm_y.ptr, perm.ptr);
        else
            init_kernel<Real><<<ceil_div(count, kBlock), kBlock, 0, stream>>>(d, d.ctl, p.omega, p.theta_initial);
        nlaunch += 1;
        bool timed_out = false;
        for (int first = 1;; first = 0) {
            if (mark_begin(9) != cudaSuccess || launch_tiny(first) != cudaSuccess || mark_end() != cudaSuccess)
                return PRAQ_ERROR_CUDA;
            nlaunch += 1;
            if (cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
                cudaStreamSynchronize(stream) != cudaSuccess)
                return PRAQ_ERROR_CUDA;
            if (mirror->status) return PRAQ_ERROR_CUDA;   // the checked build caught an index
            if (mirror->terminated) break;
            if (time_limit >= 0.0 &&
                std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count() > time_limit) {
                timed_out = true;
                break;
            }
        }
        if (timed_out) {
            mirror->result_slot = 2;
            status_override = PRAQ_STATUS_TIME_LIMIT;
            return PRAQ_STATUS_TIME_LIMIT;
        }
        status_override = -100;
        return mirror->gap <= p.tolerance ? 0 : 1;
    }

    cudaError_t launch_mega() {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(unsigned(mega_grid));
        cfg.blockDim = dim3(unsigned(kBlock));
        cfg.dynamicSmemBytes = 0;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;   // every CTA resident at once, or no launch
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const MegaArgs a{bar.ptr, unsigned(mega_grid) + mega_phantom, mega_wait_ns, nb_node, nb_edge};
        if (wide) return cudaLaunchKernelEx(&cfg, mega_block_kernel<Real, true>, d, prm, a);
        return cudaLaunchKernelEx(&cfg, mega_block_kernel<Real, false>, d, prm, a);
    }
    long long block_launches() const { return mega ? 1 : block_nodes + (exec && gated ? 1 : 0); }

    int layout(const PraqInstance& in) {
        n = int(in.n);
        m = int(in.m);
        PoolBuf<int64_t> rows, cols;
        PoolBuf<double> vals, dg, part;
        PoolBuf<int> krow, kcol, first, second, sidx, flags, keys2, iota, ksorted;
        PoolBuf<unsigned char> temp;
        if (upload_input(dg, in.diag, n) || upload_input(rows, in.rows, m) ||
            upload_input(cols, in.cols, m) || upload_input(vals, in.vals, m) ||
            krow.alloc(m, stream) || kcol.alloc(m, stream) || flags.alloc(1, stream) ||
            part.alloc(kPrepBlocks, stream) || scale.alloc(1, stream))
            return PRAQ_ERROR_CUDA;
        if (cudaMemsetAsync(flags.ptr, 0, sizeof(int), stream)) return PRAQ_ERROR_CUDA;
        prep_scan_kernel<<<kPrepBlocks, kBlock, 0, stream>>>(n, m, rows.ptr, cols.ptr, vals.ptr, dg.ptr,
                                                            krow.ptr, kcol.ptr, flags.ptr, part.ptr);
        prep_scale_kernel<<<1, kBlock, 0, stream>>>(part.ptr, kPrepBlocks, scale.ptr);
        int fl = 0;
        if (m <= kHostCheckEdges) {
            // a small instance: the same two facts from the caller's arrays on
            // the host, instead of a round trip that waits for the device
            for (int64_t e = 0; e < m; ++e) {
                const int64_t i = in.rows[e], j = in.cols[e];
                if (i < 0 || i >= n || j < 0 || j >= n || i == j) fl |= 1;
                if (e > 0 && in.rows[e - 1] > i) fl |= 2;
            }
        } else {
            int* hflags = reinterpret_cast<int*>(mirror);   // the pinned slot, before it is a mirror
            *hflags = 0;
            if (cudaMemcpyAsync(hflags, flags.ptr, sizeof(int), cudaMemcpyDeviceToHost, stream) ||
                cudaStreamSynchronize(stream))
                return PRAQ_ERROR_CUDA;
            fl = *hflags;
        }
        if (fl & 1) return PRAQ_ERROR_INSTANCE;
        if (ends.alloc(m, stream) || w.alloc(m, stream) || first.alloc(m, stream) ||
            second.alloc(m, stream) || sidx.alloc(m, stream) || row_ptr.alloc(size_t(n) + 1, stream) ||
            col_ptr.alloc(size_t(n) + 1, stream) || colidx.alloc(m, stream) || diag.alloc(n, stream) ||
            deg.alloc(n, stream) || keys2.alloc(m, stream))
            return PRAQ_ERROR_CUDA;
        int key_bits = 1;
        while (key_bits < 31 && (1LL << key_bits) < (long long)n) ++key_bits;
        auto radix = [&](const int* kin, int* kout, const int* vin, int* vout) -> int {
            size_t bytes = 0;
            if (cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, m, 0, key_bits, stream))
                return PRAQ_ERROR_CUDA;
            if (temp.count < bytes && temp.alloc(bytes, stream)) return PRAQ_ERROR_CUDA;
            if (cub::DeviceRadixSort::SortPairs(temp.ptr, bytes, kin, kout, vin, vout, m, 0, key_bits, stream))
                return PRAQ_ERROR_CUDA;
            return 0;
        };
        const int* permp = nullptr;
        if ((fl & 2) && m > 0) {
            // stable sort of the input edges by first end: perm[s] = input edge
            if (iota.alloc(m, stream) || ksorted.alloc(m, stream) || perm.alloc(m, stream))
                return PRAQ_ERROR_CUDA;
            iota_kernel<<<ceil_div(m, kBlock), kBlock, 0, stream>>>(m, iota.ptr);
            if (radix(krow.ptr, ksorted.ptr, iota.ptr, perm.ptr)) return PRAQ_ERROR_CUDA;
            permp = perm.ptr;
        }
        if (m > 0) {
            prep_edges_kernel<Real><<<ceil_div(m, kBlock), kBlock, 0, stream>>>(
                m, permp, krow.ptr, kcol.ptr, vals.ptr, scale.ptr, ends.ptr, w.ptr, first.ptr,
                second.ptr, sidx.ptr);
            // second-end order: a stable sort of the sorted edges by second end
            if (radix(second.ptr, keys2.ptr, sidx.ptr, colidx.ptr)) return PRAQ_ERROR_CUDA;
            if (!pull) {   // push: the inverse permutation, and no index afterwards
                if (colpos.alloc(m, stream)) return PRAQ_ERROR_CUDA;
                prep_colpos_kernel<<<ceil_div(m, kBlock), kBlock, 0, stream>>>(m, colidx.ptr, colpos.ptr);
                colidx.release();
            }
        }
        prep_runs_kernel<<<ceil_div((long long)n + 1, kBlock), kBlock, 0, stream>>>(n, m, first.ptr, row_ptr.ptr);
        prep_runs_kernel<<<ceil_div((long long)n + 1, kBlock), kBlock, 0, stream>>>(n, m, keys2.ptr, col_ptr.ptr);
        prep_nodes_kernel<Real><<<ceil_div(n, kBlock), kBlock, 0, stream>>>(n, row_ptr.ptr, col_ptr.ptr, dg.ptr,
                                                                          scale.ptr, diag.ptr, deg.ptr);
        return cudaGetLastError() == cudaSuccess ? 0 : PRAQ_ERROR_CUDA;
    }

    // --- profiling: an event pair around every kernel, by kind ------------
    static constexpr int kKinds = 10;   // the graph's nine kinds; a persistent-kernel block
    std::vector<cudaEvent_t> evpool;
    std::vector<std::pair<int, int>> marks;   // (kind, first event index)
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

#define RB_TIMED(kind, launch)               \
    do {                                     \
        RB_CUDA_TRY(mark_begin(kind));       \
        launch;                              \
        RB_CUDA_TRY(mark_end());             \
    } while (0)

    // One op_steps block: op_steps reflected steps (the last with the check
    // sums), the lower-bound pass, the check, then the restart step (gated on
    // the device flag), its error, and a copy of the control block to the host.
    cudaError_t enqueue_block() {
        if (mega) {
            RB_TIMED(9, RB_CUDA_TRY(launch_mega()));
            return cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream);
        }
        if (pull) return wide ? enqueue_steps<true, true>() : enqueue_steps<false, true>();
        return wide ? enqueue_steps<true, false>() : enqueue_steps<false, false>();
    }

    template <bool W, bool P>
    cudaError_t enqueue_steps() {
        const int op = int(p.op_steps);
        for (int s = 0; s < op; ++s) {
            if (s + 1 < op) {
                RB_TIMED(0, RB_CUDA_TRY(launch_pdl(node_kernel<Real, true, false, W, P>, nb_node, kBlock, stream, d, (const Real*)d.pred, (const Real*)d.pred1, s, 0, 0)));
                if (m) RB_TIMED(1, RB_CUDA_TRY(launch_pdl(edge_plain_kernel<Real, P>, P ? nb_edge_pull : nb_edge_push, kBlock, stream, d, (const Real*)nullptr, s, 0, 0)));
            } else {
                RB_TIMED(2, RB_CUDA_TRY(launch_pdl(node_kernel<Real, true, true, W, P>, nb_node, kBlock, stream, d, (const Real*)d.pred, (const Real*)d.pred1, s, 0, 0)));
                if (m) RB_TIMED(3, RB_CUDA_TRY(launch_pdl(edge_kernel<Real, true, true, P>, nb_edge, kBlock, stream, d, (const Real*)nullptr, s, 0, 0)));
            }
        }
        RB_TIMED(4, RB_CUDA_TRY(launch_pdl(lower_kernel<Real, W, P>, nb_node, kBlock, stream, d, (const Real*)d.u2s, (const Real*)d.u2s1)));
        RB_TIMED(5, RB_CUDA_TRY(launch_pdl(check_kernel, 1, kCheckBlock, stream, d.ctl, prm, (const double*)d.scale, (const double*)d.pnode, nb_node,
                                                                d.pedge, nb_edge, d.plower, nb_node, 1)));
        RB_TIMED(6, RB_CUDA_TRY(launch_pdl(node_kernel<Real, false, true, W, P>, nb_node, kBlock, stream, d, (const Real*)d.u2s, (const Real*)d.u2s1, 0, 0, 1)));
        if (m) RB_TIMED(7, RB_CUDA_TRY(launch_pdl(edge_kernel<Real, false, true, P>, nb_edge, kBlock, stream, d, (const Real*)d.u2s, 0, 0, 1)));
        RB_TIMED(8, RB_CUDA_TRY(launch_pdl(check_kernel, 1, kCheckBlock, stream, d.ctl, prm, (const double*)d.scale, (const double*)d.pnode, nb_node,
                                                                d.pedge, nb_edge, d.plower, nb_node, 2)));
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

    // The start point of later runs: x [n] and dual pairs y2 [2m] (instance
    // units, the input's edge order, as result() returns them); either may be
    // null (x = 1/2, the centroid).  Both null: back to the cold start.
    int set_warm(const double* x, const double* y2) override {
        warm_x.release();
        warm_y.release();
        if (x && warm_x.upload(x, size_t(n), stream)) return PRAQ_ERROR_CUDA;
        if (y2 && m && warm_y.upload(y2, size_t(2) * m, stream)) return PRAQ_ERROR_CUDA;
        return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : PRAQ_ERROR_CUDA;
    }

    // x1, y1 = _raw_step(x0, y0): one vanilla step from the start, with the
    // sums for the error and the bounds at the start point
    template <bool P>
    void start_step() {
        node_kernel<Real, false, true, false, P><<<nb_node, kBlock, 0, stream>>>(d, d.pred, d.pred1, 0, 1, 0);
        lower_kernel<Real, false, P><<<nb_node, kBlock, 0, stream>>>(d, d.pred, d.pred1);
        if (m) edge_kernel<Real, false, true, P><<<nb_edge, kBlock, 0, stream>>>(d, d.pred, 0, 1, 0);
    }

    // Host -> device copy of one of the caller's (pageable) instance arrays:
    // an array of at least kRingUploadBytes goes through the library's pinned
    // staging ring (host threads fill one slot while the copy engine drains
    // the other), a smaller one by the driver's own pageable copy, whose
    // rate varies from host to host (B200 boxes of one pool: 7.7 to 20 GB/s
    // pageable against 21 to 51 GB/s pinned).  REFORM_PRAQ_UPLOAD=staged|direct
    // in the environment sends every array one way (for measurements).
    static constexpr size_t kRingUploadBytes = size_t(1) << 20;
    template <class T>
    cudaError_t upload_input(PoolBuf<T>& b, const T* host, size_t count) {
        const char* env = std::getenv("REFORM_PRAQ_UPLOAD");
        const bool direct = env && !std::strcmp(env, "direct");
        const bool staged = env && !std::strcmp(env, "staged");
        if (direct || (!staged && sizeof(T) * count < kRingUploadBytes)) return b.upload(host, count, stream);
        RB_CUDA_TRY(b.alloc(count, stream));
        return staged_upload(b.ptr, host, sizeof(T) * count, stream);
    }

    // Slot-1 layout for m edges: pull once the step's edge arrays (ends, w,
    // pred, pred1, u0 and the index: 12 + 4 R bytes per edge) exceed twice the
    // L2 size.  REFORM_PRAQ_SLOT1=push|pull in the environment overrides the
    // choice (for tests and measurements).
    bool choose_pull(int64_t m_) const {
        if (!allow_pull) return false;
        const char* env = std::getenv("REFORM_PRAQ_SLOT1");
        if (env && !std::strcmp(env, "push")) return false;
        if (env && !std::strcmp(env, "pull")) return true;
        if (kPull != 2) return kPull == 1;
        int l2 = 0;
        if (once_per_device(&l2, [](int* v) {
                int dev = 0;
                RB_CUDA_TRY(cudaGetDevice(&dev));
                return cudaDeviceGetAttribute(v, cudaDevAttrL2CacheSize, dev);
            }) != cudaSuccess)
            return false;
        return double(m_) * (12.0 + 4.0 * sizeof(Real)) > 2.0 * double(l2);
    }

    // Cold (or warm) start, the first vanilla step and the check before the loop.
    int start_solve() {
        nlaunch = 0;
        if (mega && cudaMemsetAsync(bar.ptr, 0, sizeof(GridBar), stream) != cudaSuccess) return PRAQ_ERROR_CUDA;
        const int count = std::max(n, m);
        if (warm_x.ptr || warm_y.ptr)
            warm_init_kernel<Real><<<ceil_div(count, kBlock), kBlock, 0, stream>>>(
                d, d.ctl, p.omega, p.theta_initial, warm_x.ptr, warm_y.ptr, perm.ptr);
        else
            init_kernel<Real><<<ceil_div(count, kBlock), kBlock, 0, stream>>>(d, d.ctl, p.omega, p.theta_initial);
        // x1, y1 = _raw_step(x0, y0): one vanilla step from the start, with
        // the sums for the error and the bounds at the start point.
        if (pull) start_step<true>();
        else start_step<false>();
        check_kernel<<<1, kCheckBlock, 0, stream>>>(d.ctl, prm, d.scale, d.pnode, nb_node, d.pedge, nb_edge,
                                                   d.plower, nb_node, 0);
        if (cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
            return PRAQ_ERROR_CUDA;
        nlaunch += 4 + (m ? 1 : 0);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(stream) != cudaSuccess)
            return PRAQ_ERROR_CUDA;
        return 0;
    }

    int run() override {
        const auto started = std::chrono::steady_clock::now();
        if (tiny) return run_tiny(started);
        bool timed_out = false;
        // the first run launches directly; repeated runs replay a captured block
        if (runs++ > 0 && !exec && !mega && capture_block() != cudaSuccess) return PRAQ_ERROR_CUDA;
        {
            const int st = start_solve();
            if (st) return st;
        }
        // Keep one block in flight ahead of the one being inspected; blocks
        // launched after termination see the flag and return at once.
        if (!mirror->terminated) {
            for (int k = 0; k < 2; ++k) {
                if (launch_block() != cudaSuccess) return PRAQ_ERROR_CUDA;
                if (cudaEventRecord(done[k], stream) != cudaSuccess) return PRAQ_ERROR_CUDA;
                nlaunch += block_launches();
            }
            int k = 0;
            for (;;) {
                if (cudaEventSynchronize(done[k]) != cudaSuccess) return PRAQ_ERROR_CUDA;
                if (mirror->terminated && !mirror->status && exec && gated && !mega)
                    nlaunch -= block_nodes;   // the block behind it ran its gate alone
                if (mirror->status || mirror->terminated) break;
                if (time_limit >= 0.0 &&
                    std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count() >
                        time_limit) {
                    timed_out = true;
                    break;
                }
                if (launch_block() != cudaSuccess) return PRAQ_ERROR_CUDA;
                if (cudaEventRecord(done[k], stream) != cudaSuccess) return PRAQ_ERROR_CUDA;
                nlaunch += block_launches();
                k ^= 1;
            }
        }
        if (cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess)
            return PRAQ_ERROR_CUDA;
        if (mirror->status) return PRAQ_ERROR_CUDA;   // a barrier of the persistent kernel ran out
        if (timed_out && !mirror->terminated) {
            mirror->result_slot = 2;
            status_override = PRAQ_STATUS_TIME_LIMIT;
            return PRAQ_STATUS_TIME_LIMIT;
        }
        status_override = -100;
        return mirror->gap <= p.tolerance ? 0 : 1;
    }

    // A solve with every kernel launched on its own (no graph) between an
    // event pair; each kind's total milliseconds and launch count go to
    // ms[kKinds], count[kKinds].  Same arithmetic; the host waits after every
    // block.
    int run_profiled(double* ms, long long* count) override {
        for (int k = 0; k < kKinds; ++k) { ms[k] = 0.0; count[k] = 0; }
        if (tiny) {   // each launch of the single-CTA form as one mark of kind 9
            marks.clear();
            profiling = true;
            const double budget = time_limit;
            time_limit = -1.0;
            const int st = run_tiny(std::chrono::steady_clock::now());
            time_limit = budget;
            profiling = false;
            if (st < 0) return st;
            for (auto& mk : marks) {
                float t = 0.f;
                if (cudaEventElapsedTime(&t, evpool[mk.second], evpool[mk.second + 1]) != cudaSuccess)
                    return PRAQ_ERROR_CUDA;
                ms[mk.first] += t;
                count[mk.first] += 1;
            }
            return st;
        }
        int st = start_solve();
        if (st) return st;
        profiling = true;
        while (!mirror->terminated) {
            marks.clear();
            if (enqueue_block() != cudaSuccess || cudaStreamSynchronize(stream) != cudaSuccess) {
                profiling = false;
                return PRAQ_ERROR_CUDA;
            }
            nlaunch += block_launches();
            if (mirror->status) {
                profiling = false;
                return PRAQ_ERROR_CUDA;
            }
            for (auto& mk : marks) {
                float t = 0.f;
                if (cudaEventElapsedTime(&t, evpool[mk.second], evpool[mk.second + 1]) != cudaSuccess) {
                    profiling = false;
                    return PRAQ_ERROR_CUDA;
                }
                ms[mk.first] += t;
                count[mk.first] += 1;
            }
        }
        profiling = false;
        if (cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess)
            return PRAQ_ERROR_CUDA;
        status_override = -100;
        return mirror->gap <= p.tolerance ? 0 : 1;
    }

    int result(double* x, double* y2, PraqResult* res) override {
        const Control c = *mirror;
        if (x) {
            const Real* src = c.result_slot == 1 ? d.x1 : d.x2;
            // through the library's pinned ring (no ring to be had: a host
            // vector and the driver's pageable copy)
            const cudaError_t st = staged_download_as_double(x, src, size_t(n), stream);
            if (st == cudaErrorMemoryAllocation) {
                std::vector<Real> hx(n);
                if (cudaMemcpyAsync(hx.data(), src, sizeof(Real) * n, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
                    cudaStreamSynchronize(stream) != cudaSuccess)
                    return PRAQ_ERROR_CUDA;
                for (int i = 0; i < n; ++i) x[i] = double(hx[i]);
            } else if (st != cudaSuccess) {
                return PRAQ_ERROR_CUDA;
            }
        }
        if (y2 && m) {
            std::vector<Real> hu(m), hw(m);
            std::vector<int> hp(perm.ptr ? m : 0);
            double sc = 1.0;
            const Real* src = c.result_slot == 1 ? d.u0 : d.u2s;
            if (cudaMemcpyAsync(hu.data(), src, sizeof(Real) * m, cudaMemcpyDeviceToHost, stream) ||
                cudaMemcpyAsync(hw.data(), d.w, sizeof(Real) * m, cudaMemcpyDeviceToHost, stream) ||
                cudaMemcpyAsync(&sc, d.scale, sizeof(double), cudaMemcpyDeviceToHost, stream) ||
                (perm.ptr && cudaMemcpyAsync(hp.data(), perm.ptr, sizeof(int) * m, cudaMemcpyDeviceToHost, stream)) ||
                cudaStreamSynchronize(stream))
                return PRAQ_ERROR_CUDA;
            for (int s = 0; s < m; ++s) {
                const int e = perm.ptr ? hp[s] : s;
                const double u = double(hu[s]), sw = double(hw[s]);
                y2[2 * e] = u * sc;
                y2[2 * e + 1] = (sw > 0.0 ? u : (-sw - u)) * sc;
            }
        }
        if (res) {
            res->lower = c.lower;
            res->upper = c.upper;
            res->iterations = c.iteration;
            res->status = status_override != -100 ? status_override : (c.gap <= p.tolerance ? 0 : 1);
        }
        return 0;
    }

    long long launches() const override { return nlaunch; }

    // The trace ring lives in the check parameters, which a captured block
    // holds by value: a new ring drops the capture, the next run makes one.
    int set_trace(int capacity) override {
        if (cudaStreamSynchronize(stream) != cudaSuccess) return PRAQ_ERROR_CUDA;
        trace.release();
        prm.trace = nullptr;
        prm.trace_cap = 0;
        if (capacity > 0) {
            if (trace.alloc(size_t(capacity), stream) != cudaSuccess) return PRAQ_ERROR_CUDA;
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
        if (cudaMemcpyAsync(ring.data(), prm.trace, sizeof(reform_trace_record) * ring.size(), cudaMemcpyDeviceToHost,
                            stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess)
            return PRAQ_ERROR_CUDA;
        const long long count = std::min<long long>({len, (long long)prm.trace_cap, (long long)capacity});
        for (long long k = 0; k < count; ++k) out[k] = ring[size_t((len - count + k) % prm.trace_cap)];
        return 0;
    }

    size_t device_bytes() const {
        size_t b = 0;
        b += (row_ptr.count + col_ptr.count + colidx.count + colpos.count + perm.count) * sizeof(int);
        b += ends.count * sizeof(int2);
        for (auto* x : {&w, &diag, &deg, &x1, &x2, &x0, &r, &pred, &pred1, &u0, &u2s, &u2s1})
            b += x->count * sizeof(Real);
        for (auto* x : {&pnode, &pedge, &plower, &scale}) b += x->count * sizeof(double);
        return b + sizeof(Control);
    }
};

static bool valid(const PraqParameters& p) {
    return p.tolerance >= 0.0 && p.omega > 0.0 && p.beta_sufficient > 0.0 &&
           p.beta_necessary > 0.0 && p.beta_artificial >= 0.0 && std::isfinite(p.theta_initial) &&
           std::isfinite(p.theta_target) && std::isfinite(p.theta_decay) &&
           std::isfinite(p.interval_offset) && std::isfinite(p.interval_scale) &&
           p.interval_power >= 0.0;
}

}  // namespace
}  // namespace praq
}  // namespace rb200
