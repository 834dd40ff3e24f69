// praq_solver.cu -- PRAQ (QUBO roof-dual LP) on B200: restarted, reflected
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
//   carried as the single coordinate u (mu, or a).  The per-edge projection
//   of y + eta omega (q - S r) then collapses to
//       covering:  mu' = clip(mu + (eta omega / 2)(1 - r_i - r_j), -w, 0)
//       packing:   a'  = clip(a  + (eta omega / 2)(r_j - r_i),      0, w)
//   and the scatter S^T y at node v is the sum of u over the edges where v is
//   the first end, plus the sum of +u (covering) or -u (packing) over the
//   edges where v is the second end, plus the constant sum of w over those
//   packing edges (precomputed per node).
// * Edges sorted by first end (stable counting sort), so a node's first-end
//   half-edges are one contiguous run of `pred`, read without an index; the
//   second-end half-edges come through a CSC index whose sign bit carries the
//   covering/packing sign.  Deterministic: every sum has a fixed order that
//   depends on the instance and the launch shape only.
// * `pred` holds the NEXT step's Halpern-combined dual, computed by the edge
//   kernel as it finishes a step (as the reference does), so a reflected step
//   reads one real per edge for the dual instead of three.
// * Every decision of _halpern_step (restart tests, omega/theta update,
//   termination) runs on the device in `check_kernel`, so one op_steps block
//   (op_steps x (node, edge) + check + the conditional restart step) is one
//   captured CUDA graph, replayed with no host inputs.  The host keeps one
//   block in flight ahead of the one it inspects.
//
// Launch shapes: node kernels use `lanes` consecutive lanes per node (the
// smallest power of two giving <= 8 half-edges per lane, at most 32, as
// qubo/praq-cuda/src/solver.cuh:602-614 sizes it), 256 threads per block;
// edge kernels one edge per thread; checks are one 256-thread block.
#include "../../include/praq.h"
#include "common.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>

namespace rb200 {
namespace praq {

constexpr double kEta = 0.999;   // 0.999 / ||A||_2, ||A||_2 = 1 for the half-edge lift
constexpr int kBlock = 256;
constexpr int kNodeSums = 3;     // sum deg (x1-x2)^2, sum deg (x1-x0)^2, sum d . bx
constexpr int kEdgeSums = 5;     // sum |y1-y2|^2, <S(x1-x2), y1-y2>, sum |y1-y0|^2,
                                 // upper edge term at bx, sum of covering by_1
constexpr int kCheckBlock = 256;

// Scalar state of the solve (StepArguments' scalars, solver.py:229-256),
// resident on the device.
struct Control {
    double omega, theta, fp_error, check_error;
    double new_error, lower, upper, gap;
    long long restart_iter, iteration;
    int terminated;   // the loop is over
    int restart;      // the restart step of this block is pending
    int result_slot;  // 1: (x1, u1) hold the returned point, 2: (x2, u2s)
    int status;
};

struct Params {
    double tolerance;
    long long max_iter, op_steps;
    double beta_sufficient, beta_necessary, beta_artificial;
    double theta_target, theta_decay;
    double scale;
};

template <class Real>
struct Dev {
    int n, m, lanes, lane_shift;
    const int* row_ptr;    // [n+1] first-end runs in edge order
    const int* col_ptr;    // [n+1] second-end runs in col_idx
    const int* col_idx;    // [m] edge index, bitwise NOT for packing edges
    const int2* ends;      // [m]
    const Real* w;         // [m] signed, 2 W_ij / scale
    const Real* diag;      // [n] W_ii / scale
    const Real* deg;       // [n] incident half-edges, floored at 1
    const Real* cpack;     // [n] sum of w over packing edges with this second end
    Real *x1, *x2, *x0, *r;
    Real *pred, *u0, *u2s;
    double *pnode, *pedge, *plower;
    Control* ctl;
};

template <class Real>
__device__ __forceinline__ bool skip(const Control* c, int gate) {
    return c->terminated || (gate && !c->restart);
}

// Gather S^T y at node i for a group of `lanes` lanes (sum over the group,
// every lane ends with the same bits).  All lanes of the warp must call it.
template <class Real, class Acc>
__device__ __forceinline__ Acc scatter_at(const Dev<Real>& d, const Real* __restrict__ src,
                                          long long i, int lane) {
    Acc s = Acc(0);
    if (i < d.n) {
        const int a = d.row_ptr[i], b = d.row_ptr[i + 1];
        for (int k = a + lane; k < b; k += d.lanes) s += Acc(src[k]);
        const int c0 = d.col_ptr[i], c1 = d.col_ptr[i + 1];
        for (int k = c0 + lane; k < c1; k += d.lanes) {
            const int e = d.col_idx[k];
            s += e >= 0 ? Acc(src[e]) : -Acc(src[~e]);
        }
    }
    for (int o = d.lanes >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// Primal half of one PDHG step, with the Halpern combination of x folded in
// (solver.py:259-267 and 276-292).  Reflect: x1 = lw (2 x2 - x1) + rw x0 with
// k = restart_iter + step + 1; vanilla: x1 = x2 and the anchor becomes x1.
// Check: add the node sums of this step to pnode.
template <class Real, bool Reflect, bool Check>
__global__ void __launch_bounds__(kBlock)
node_kernel(Dev<Real> d, const Real* __restrict__ ysrc, int step, int bounds_at_1, int gate) {
    const Control* c = d.ctl;
    if (skip<Real>(c, gate)) return;
    __shared__ double scratch[kNodeSums * 32];
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & (d.lanes - 1);
    const long long i = g >> d.lane_shift;
    const Real* src = Reflect ? d.pred : ysrc;
    Real s = scatter_at<Real, Real>(d, src, i, lane);
    double acc[kNodeSums] = {0.0, 0.0, 0.0};
    if (i < d.n && lane == 0) {
        s += d.cpack[i];
        const Real x2o = d.x2[i];
        Real x1v;
        if (Reflect) {
            const double k = double(c->restart_iter + step + 1);
            const Real lw = Real(k / (k + 1.0)), rw = Real(1.0 / (k + 1.0));
            x1v = lw * (Real(2) * x2o - d.x1[i]) + rw * d.x0[i];
        } else {
            x1v = x2o;
        }
        const Real ps = Real(kEta / c->omega);
        const Real grad = d.diag[i] - s;
        const Real x2v = clampv(x1v - ps * (grad / d.deg[i]), Real(0), Real(1));
        d.x1[i] = x1v;
        d.x2[i] = x2v;
        d.r[i] = Real(2) * x2v - x1v;
        if (!Reflect) d.x0[i] = x1v;
        if (Check) {
            const double deg = double(d.deg[i]);
            const double dx = double(x1v) - double(x2v);
            const double dr = double(x1v) - double(Reflect ? d.x0[i] : x1v);
            acc[0] = deg * dx * dx;
            acc[1] = deg * dr * dr;
            acc[2] = double(d.diag[i]) * double(bounds_at_1 ? x1v : x2v);
        }
    }
    if (Check) {
        block_sums<kNodeSums>(acc, scratch, acc);
        if (threadIdx.x == 0) {
            for (int k = 0; k < kNodeSums; ++k) d.pnode[size_t(blockIdx.x) * kNodeSums + k] = acc[k];
        }
    }
}

// Dual half of one PDHG step (solver.py:269-273, projection.py:16-42) in the
// one-coordinate form, plus the prediction of the next step's combined dual.
template <class Real, bool Reflect, bool Check>
__global__ void __launch_bounds__(kBlock)
edge_kernel(Dev<Real> d, const Real* __restrict__ ysrc, int step, int bounds_at_1, int gate) {
    const Control* c = d.ctl;
    if (skip<Real>(c, gate)) return;
    __shared__ double scratch[kEdgeSums * 32];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[kEdgeSums] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (e < d.m) {
        const int2 ij = d.ends[e];
        const Real sw = d.w[e];
        const bool cov = sw > Real(0);
        const Real w = cov ? sw : -sw;
        const Real u1 = Reflect ? d.pred[e] : ysrc[e];
        const Real u0 = Reflect ? d.u0[e] : u1;
        const Real ri = d.r[ij.x], rj = d.r[ij.y];
        const Real hs = Real(0.5 * kEta * c->omega);
        const Real u2 = cov ? clampv(u1 + hs * ((Real(1) - ri) - rj), -w, Real(0))
                            : clampv(u1 + hs * (rj - ri), Real(0), w);
        const double kn = Reflect ? double(c->restart_iter + step + 2) : 1.0;
        const Real lwn = Real(kn / (kn + 1.0)), rwn = Real(1.0 / (kn + 1.0));
        d.pred[e] = lwn * (Real(2) * u2 - u1) + rwn * u0;
        if (!Reflect) d.u0[e] = u1;
        if (Check) {
            d.u2s[e] = u2;
            const double x1i = d.x1[ij.x], x2i = d.x2[ij.x];
            const double x1j = d.x1[ij.y], x2j = d.x2[ij.y];
            const double dy = double(u1) - double(u2);
            const double dxi = x1i - x2i, dxj = x1j - x2j;
            acc[0] = 2.0 * dy * dy;
            acc[1] = (cov ? dxi + dxj : dxi - dxj) * dy;
            const double dr = double(u1) - double(u0);
            acc[2] = 2.0 * dr * dr;
            const double bi = bounds_at_1 ? x1i : x2i, bj = bounds_at_1 ? x1j : x2j;
            const double wd = double(w);
            acc[3] = cov ? wd * fmax(bi + bj - 1.0, 0.0) : -wd * fmin(bi, bj);
            acc[4] = cov ? double(bounds_at_1 ? u1 : u2) : 0.0;
        }
    }
    if (Check) {
        block_sums<kEdgeSums>(acc, scratch, acc);
        if (threadIdx.x == 0) {
            for (int k = 0; k < kEdgeSums; ++k) d.pedge[size_t(blockIdx.x) * kEdgeSums + k] = acc[k];
        }
    }
}

// The node part of the lower bound, sum_i min(d_i - (S^T y)_i, 0), at the
// dual `ysrc` (solver.py:333-337), accumulated in FP64.
template <class Real>
__global__ void __launch_bounds__(kBlock) lower_kernel(Dev<Real> d, const Real* __restrict__ ysrc) {
    const Control* c = d.ctl;
    if (c->terminated) return;
    __shared__ double scratch[32];
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & (d.lanes - 1);
    const long long i = g >> d.lane_shift;
    double s = scatter_at<Real, double>(d, ysrc, i, lane);
    double acc[1] = {0.0};
    if (i < d.n && lane == 0) {
        const double rc = double(d.diag[i]) - (s + double(d.cpack[i]));
        acc[0] = rc < 0.0 ? rc : 0.0;
    }
    block_sums<1>(acc, scratch, acc);
    if (threadIdx.x == 0) d.plower[blockIdx.x] = acc[0];
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
__global__ void __launch_bounds__(kCheckBlock)
check_kernel(Control* c, Params p, const double* __restrict__ pnode, int nbn,
             const double* __restrict__ pedge, int nbe, const double* __restrict__ plower,
             int nbl, int mode) {
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
    const double upper = (node[2] + edge[3]) * p.scale;
    const double lower = (low[0] + edge[4]) * p.scale;
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
        const Real u = Real(-0.5) * d.w[k];
        d.u0[k] = u;
        d.pred[k] = u;
        d.u2s[k] = u;
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
    }
}

// ---------------------------------------------------------------------------
// host side

struct HostLayout {
    int n = 0, m = 0;
    double scale = 1.0;
    std::vector<int> row_ptr, col_ptr, col_idx, perm;   // perm: sorted -> input edge
    std::vector<int2> ends;
    std::vector<double> w, diag, deg, cpack;
};

// Validation (qubo/praq-cuda/src/praq.cu:35-79, solver.cuh:524-538) and the
// device layout.  Returns 0 or PRAQ_ERROR_INSTANCE.
static int build_layout(const PraqInstance& in, HostLayout& L) {
    const int64_t limit = std::numeric_limits<int>::max();
    if (in.n <= 0 || in.n > limit / 32 || in.m < 0 || in.m > limit / 2) return PRAQ_ERROR_INSTANCE;
    if (!in.diag || (in.m > 0 && (!in.rows || !in.cols || !in.vals))) return PRAQ_ERROR_INSTANCE;
    const int n = int(in.n), m = int(in.m);
    for (int e = 0; e < m; ++e) {
        const int64_t i = in.rows[e], j = in.cols[e];
        if (i < 0 || i >= in.n || j < 0 || j >= in.n || i == j) return PRAQ_ERROR_INSTANCE;
    }
    L.n = n;
    L.m = m;
    double squares = 0.0;
    for (int i = 0; i < n; ++i) squares += in.diag[i] * in.diag[i];
    for (int e = 0; e < m; ++e) squares += 4.0 * in.vals[e] * in.vals[e];
    L.scale = squares > 0.0 ? std::sqrt(squares) : 1.0;

    // stable counting sort of edges by first end
    L.row_ptr.assign(n + 1, 0);
    for (int e = 0; e < m; ++e) ++L.row_ptr[in.rows[e] + 1];
    for (int i = 0; i < n; ++i) L.row_ptr[i + 1] += L.row_ptr[i];
    L.perm.resize(m);
    {
        std::vector<int> fill(L.row_ptr.begin(), L.row_ptr.end() - 1);
        for (int e = 0; e < m; ++e) L.perm[fill[in.rows[e]]++] = e;
    }
    L.ends.resize(m);
    L.w.resize(m);
    for (int s = 0; s < m; ++s) {
        const int e = L.perm[s];
        L.ends[s] = make_int2(int(in.rows[e]), int(in.cols[e]));
        L.w[s] = 2.0 * in.vals[e] / L.scale;
    }
    // second-end runs, edges in increasing sorted order inside each run
    L.col_ptr.assign(n + 1, 0);
    for (int s = 0; s < m; ++s) ++L.col_ptr[L.ends[s].y + 1];
    for (int i = 0; i < n; ++i) L.col_ptr[i + 1] += L.col_ptr[i];
    L.col_idx.resize(m);
    L.cpack.assign(n, 0.0);
    {
        std::vector<int> fill(L.col_ptr.begin(), L.col_ptr.end() - 1);
        for (int s = 0; s < m; ++s) {
            const int j = L.ends[s].y;
            const bool cov = L.w[s] > 0.0;
            L.col_idx[fill[j]++] = cov ? s : ~s;
            if (!cov) L.cpack[j] += -L.w[s];   // w = |signed w|
        }
    }
    L.diag.resize(n);
    L.deg.resize(n);
    for (int i = 0; i < n; ++i) {
        L.diag[i] = in.diag[i] / L.scale;
        const int incident = (L.row_ptr[i + 1] - L.row_ptr[i]) + (L.col_ptr[i + 1] - L.col_ptr[i]);
        L.deg[i] = incident > 0 ? double(incident) : 1.0;
    }
    return 0;
}

static int lanes_for(int n, int m) {
    const double average = 2.0 * double(m) / double(n);
    int lanes = 1;
    while (lanes < 32 && double(lanes) * 8.0 < average) lanes *= 2;
    return lanes;
}

struct SolverBase {
    virtual ~SolverBase() = default;
    virtual int run() = 0;
    virtual int result(double* x, double* y2, PraqResult* r) = 0;
    virtual long long launches() const = 0;
    virtual int run_profiled(double* ms, long long* count) = 0;
    double time_limit = -1.0;   // seconds of wall clock per run; < 0: none
};

template <class Real>
struct Solver final : SolverBase {
    HostLayout L;
    Params prm{};
    PraqParameters p{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    DevBuf<int> row_ptr, col_ptr, col_idx;
    DevBuf<int2> ends;
    DevBuf<Real> w, diag, deg, cpack, x1, x2, x0, r, pred, u0, u2s;
    DevBuf<double> pnode, pedge, plower;
    DevBuf<Control> ctl;
    Control* mirror = nullptr;   // pinned host copy of the control block
    Dev<Real> d{};
    int nb_node = 1, nb_edge = 1;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t done[2] = {nullptr, nullptr};
    long long nlaunch = 0, block_nodes = 0;
    int status_override = -100;

    ~Solver() override {
        if (stream) cudaStreamSynchronize(stream);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto& ev : done) if (ev) cudaEventDestroy(ev);
        for (auto& ev : evpool) cudaEventDestroy(ev);
        row_ptr.release(); col_ptr.release(); col_idx.release(); ends.release();
        w.release(); diag.release(); deg.release(); cpack.release();
        x1.release(); x2.release(); x0.release(); r.release(); pred.release(); u0.release();
        u2s.release(); pnode.release(); pedge.release(); plower.release(); ctl.release();
        if (stream) cudaStreamSynchronize(stream);
        if (mirror) cudaFreeHost(mirror);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    template <class T>
    static std::vector<T> cast(const std::vector<double>& v) { return std::vector<T>(v.begin(), v.end()); }

    cudaError_t setup(cudaStream_t s) {
        if (s) {
            stream = s;
        } else {
            RB_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
            own_stream = true;
        }
        const int n = L.n, m = L.m;
        RB_CUDA_TRY(row_ptr.upload(L.row_ptr.data(), n + 1, stream));
        RB_CUDA_TRY(col_ptr.upload(L.col_ptr.data(), n + 1, stream));
        RB_CUDA_TRY(col_idx.upload(L.col_idx.data(), m, stream));
        RB_CUDA_TRY(ends.upload(L.ends.data(), m, stream));
        auto wr = cast<Real>(L.w), dr = cast<Real>(L.diag), gr = cast<Real>(L.deg),
             cr = cast<Real>(L.cpack);
        RB_CUDA_TRY(w.upload(wr.data(), m, stream));
        RB_CUDA_TRY(diag.upload(dr.data(), n, stream));
        RB_CUDA_TRY(deg.upload(gr.data(), n, stream));
        RB_CUDA_TRY(cpack.upload(cr.data(), n, stream));
        for (auto* b : {&x1, &x2, &x0, &r}) RB_CUDA_TRY(b->alloc(n, stream));
        for (auto* b : {&pred, &u0, &u2s}) RB_CUDA_TRY(b->alloc(m, stream));
        const int lanes = lanes_for(n, m);
        nb_node = ceil_div((long long)n * lanes, kBlock);
        nb_edge = std::max(1, ceil_div(m, kBlock));
        RB_CUDA_TRY(pnode.alloc(size_t(nb_node) * kNodeSums, stream));
        RB_CUDA_TRY(pedge.alloc(size_t(nb_edge) * kEdgeSums, stream));
        RB_CUDA_TRY(plower.alloc(size_t(nb_node), stream));
        RB_CUDA_TRY(ctl.alloc(1, stream));
        RB_CUDA_TRY(cudaMemsetAsync(pedge.ptr, 0, sizeof(double) * pedge.count, stream));
        RB_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&mirror), sizeof(Control)));
        for (auto& ev : done) RB_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));

        d.n = n; d.m = m; d.lanes = lanes;
        d.lane_shift = 0;
        while ((1 << d.lane_shift) < lanes) ++d.lane_shift;
        d.row_ptr = row_ptr.ptr; d.col_ptr = col_ptr.ptr; d.col_idx = col_idx.ptr;
        d.ends = ends.ptr; d.w = w.ptr; d.diag = diag.ptr; d.deg = deg.ptr; d.cpack = cpack.ptr;
        d.x1 = x1.ptr; d.x2 = x2.ptr; d.x0 = x0.ptr; d.r = r.ptr;
        d.pred = pred.ptr; d.u0 = u0.ptr; d.u2s = u2s.ptr;
        d.pnode = pnode.ptr; d.pedge = pedge.ptr; d.plower = plower.ptr; d.ctl = ctl.ptr;

        prm.tolerance = p.tolerance;
        prm.max_iter = p.max_iter;
        prm.op_steps = p.op_steps;
        prm.beta_sufficient = p.beta_sufficient;
        prm.beta_necessary = p.beta_necessary;
        prm.beta_artificial = p.beta_artificial;
        prm.theta_target = p.theta_target;
        prm.theta_decay = p.theta_decay;
        prm.scale = L.scale;
        RB_CUDA_TRY(capture_block());
        return cudaStreamSynchronize(stream);
    }

    // One op_steps block: op_steps reflected steps (the last with the check
    // sums), the lower-bound pass, the check, then the restart step (gated on
    // the device flag), its error, and a copy of the control block to the host.
    // Profiled launches: an event pair around every kernel, by kind
    // (0 node, 1 edge, 2 node+check, 3 edge+check, 4 lower, 5 check,
    // 6 restart node, 7 restart edge, 8 restart check).
    static constexpr int kKinds = 9;
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
        const int op = int(p.op_steps);
        for (int s = 0; s < op; ++s) {
            if (s + 1 < op) {
                RB_TIMED(0, (node_kernel<Real, true, false><<<nb_node, kBlock, 0, stream>>>(d, nullptr, s, 0, 0)));
                if (L.m) RB_TIMED(1, (edge_kernel<Real, true, false><<<nb_edge, kBlock, 0, stream>>>(d, nullptr, s, 0, 0)));
            } else {
                RB_TIMED(2, (node_kernel<Real, true, true><<<nb_node, kBlock, 0, stream>>>(d, nullptr, s, 0, 0)));
                if (L.m) RB_TIMED(3, (edge_kernel<Real, true, true><<<nb_edge, kBlock, 0, stream>>>(d, nullptr, s, 0, 0)));
            }
        }
        RB_TIMED(4, (lower_kernel<Real><<<nb_node, kBlock, 0, stream>>>(d, d.u2s)));
        RB_TIMED(5, (check_kernel<<<1, kCheckBlock, 0, stream>>>(d.ctl, prm, d.pnode, nb_node, d.pedge,
                                                                nb_edge, d.plower, nb_node, 1)));
        RB_TIMED(6, (node_kernel<Real, false, true><<<nb_node, kBlock, 0, stream>>>(d, d.u2s, 0, 0, 1)));
        if (L.m) RB_TIMED(7, (edge_kernel<Real, false, true><<<nb_edge, kBlock, 0, stream>>>(d, d.u2s, 0, 0, 1)));
        RB_TIMED(8, (check_kernel<<<1, kCheckBlock, 0, stream>>>(d.ctl, prm, d.pnode, nb_node, d.pedge,
                                                                nb_edge, d.plower, nb_node, 2)));
        RB_CUDA_TRY(cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream));
        return cudaGetLastError();
    }

    // A solve with every kernel launched on its own (no graph) between an
    // event pair; adds each kind's total milliseconds and launch count into
    // ms[kKinds], count[kKinds].  A measurement mode: same arithmetic, the
    // host waits after every block.
    int run_profiled(double* ms, long long* count) override {
        for (int k = 0; k < kKinds; ++k) { ms[k] = 0.0; count[k] = 0; }
        int st = start_solve();
        if (st) return st;
        profiling = true;
        while (!mirror->terminated) {
            marks.clear();
            if (enqueue_block() != cudaSuccess || cudaStreamSynchronize(stream) != cudaSuccess) {
                profiling = false;
                return PRAQ_ERROR_CUDA;
            }
            nlaunch += block_nodes;
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

    cudaError_t capture_block() {
        RB_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t st = enqueue_block();
        cudaError_t st2 = cudaStreamEndCapture(stream, &graph);
        RB_CUDA_TRY(st);
        RB_CUDA_TRY(st2);
        RB_CUDA_TRY(cudaGraphInstantiate(&exec, graph, 0));
        const int op = int(p.op_steps);
        block_nodes = (L.m ? 2 : 1) * (long long)op + 2 + (L.m ? 2 : 1) + 1;
        return cudaSuccess;
    }

    // Cold start, the first vanilla step and the check before the loop.
    int start_solve() {
        nlaunch = 0;
        const int count = std::max(L.n, L.m);
        init_kernel<Real><<<ceil_div(count, kBlock), kBlock, 0, stream>>>(d, d.ctl, p.omega,
                                                                           p.theta_initial);
        // x1, y1 = _raw_step(x0, y0): one vanilla step from the start, with
        // the sums for the error and the bounds at the start point.
        node_kernel<Real, false, true><<<nb_node, kBlock, 0, stream>>>(d, d.u0, 0, 1, 0);
        if (L.m) edge_kernel<Real, false, true><<<nb_edge, kBlock, 0, stream>>>(d, d.u0, 0, 1, 0);
        lower_kernel<Real><<<nb_node, kBlock, 0, stream>>>(d, d.u0);
        check_kernel<<<1, kCheckBlock, 0, stream>>>(d.ctl, prm, d.pnode, nb_node, d.pedge, nb_edge,
                                                   d.plower, nb_node, 0);
        if (cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
            return PRAQ_ERROR_CUDA;
        nlaunch += 4 + (L.m ? 1 : 0);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(stream) != cudaSuccess)
            return PRAQ_ERROR_CUDA;
        return 0;
    }

    int run() override {
        nlaunch = 0;
        const auto started = std::chrono::steady_clock::now();
        bool timed_out = false;
        {
            const int st = start_solve();
            if (st) return st;
        }
        // Keep one block in flight ahead of the one being inspected; blocks
        // launched after termination see the flag and return at once.
        int inflight = 0;
        if (!mirror->terminated) {
            for (int k = 0; k < 2; ++k) {
                if (cudaGraphLaunch(exec, stream) != cudaSuccess) return PRAQ_ERROR_CUDA;
                if (cudaEventRecord(done[k], stream) != cudaSuccess) return PRAQ_ERROR_CUDA;
                nlaunch += block_nodes;
                ++inflight;
            }
            int k = 0;
            for (;;) {
                if (cudaEventSynchronize(done[k]) != cudaSuccess) return PRAQ_ERROR_CUDA;
                if (mirror->terminated) break;
                if (time_limit >= 0.0 &&
                    std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count() >
                        time_limit) {
                    timed_out = true;
                    break;
                }
                if (cudaGraphLaunch(exec, stream) != cudaSuccess) return PRAQ_ERROR_CUDA;
                if (cudaEventRecord(done[k], stream) != cudaSuccess) return PRAQ_ERROR_CUDA;
                nlaunch += block_nodes;
                k ^= 1;
            }
        }
        if (cudaMemcpyAsync(mirror, d.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess)
            return PRAQ_ERROR_CUDA;
        if (timed_out && !mirror->terminated) {
            // the last completed check's bracket stands; the returned point is
            // the one it was measured at
            mirror->result_slot = 2;
            status_override = PRAQ_STATUS_TIME_LIMIT;
            return PRAQ_STATUS_TIME_LIMIT;
        }
        status_override = -100;
        return mirror->gap <= p.tolerance ? 0 : 1;
    }

    int result(double* x, double* y2, PraqResult* res) override {
        const Control c = *mirror;
        if (x) {
            std::vector<Real> hx(L.n);
            const Real* src = c.result_slot == 1 ? d.x1 : d.x2;
            if (cudaMemcpyAsync(hx.data(), src, sizeof(Real) * L.n, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
                cudaStreamSynchronize(stream) != cudaSuccess)
                return PRAQ_ERROR_CUDA;
            for (int i = 0; i < L.n; ++i) x[i] = double(hx[i]);
        }
        if (y2 && L.m) {
            std::vector<Real> hu(L.m);
            const Real* src = c.result_slot == 1 ? d.u0 : d.u2s;
            if (cudaMemcpyAsync(hu.data(), src, sizeof(Real) * L.m, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
                cudaStreamSynchronize(stream) != cudaSuccess)
                return PRAQ_ERROR_CUDA;
            for (int s = 0; s < L.m; ++s) {
                const int e = L.perm[s];
                const double u = double(hu[s]), sw = L.w[s];
                y2[2 * e] = u * L.scale;
                y2[2 * e + 1] = (sw > 0.0 ? u : (-sw - u)) * L.scale;
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
};

static bool valid(const PraqParameters& p) {
    return p.tolerance >= 0.0 && p.omega > 0.0 && p.beta_sufficient > 0.0 &&
           p.beta_necessary > 0.0 && p.beta_artificial >= 0.0 && std::isfinite(p.theta_initial) &&
           std::isfinite(p.theta_target) && std::isfinite(p.theta_decay) &&
           std::isfinite(p.interval_offset) && std::isfinite(p.interval_scale) &&
           p.interval_power >= 0.0;
}

}  // namespace praq
}  // namespace rb200

using namespace rb200;

struct reform_praq_solver {
    std::unique_ptr<praq::SolverBase> impl;
};

extern "C" {

PraqParameters praq_default_parameters(void) {
    PraqParameters p;
    p.tolerance = 1e-8;
    p.max_iter = -1;
    p.use_float32 = 0;
    p.omega = 1.0;
    p.beta_sufficient = 0.36787944117144233;   // exp(-1)
    p.beta_necessary = 0.5706;
    p.beta_artificial = 0.2468;
    p.theta_initial = 0.81930;
    p.theta_target = 0.42818;
    p.theta_decay = 0.90474;
    p.op_steps = 16;
    p.interval_offset = 0.0;
    p.interval_scale = 4.328085122666891;      // 3 / ln 2
    p.interval_power = 0.0;
    return p;
}

int64_t praq_check_interval(int64_t n, const PraqParameters* parameters) {
    if (!parameters || n <= 0) return 2;
    const double u = std::log(double(n) / 50000.0);
    const double pw = parameters->interval_power;
    const double b = pw == 0.0 ? u : std::expm1(pw * u) / pw;
    const double v = std::floor(parameters->interval_offset + parameters->interval_scale * b + 0.5);
    if (!(v >= 2.0)) return 2;
    if (v > 1e9) return 1000000000;
    return int64_t(v);
}

int reform_praq_create(const PraqInstance* instance, const PraqParameters* parameters,
                       void* stream, reform_praq_solver** out) {
    if (out) *out = nullptr;
    if (!instance || !parameters || !out) return PRAQ_ERROR_ARGUMENT;
    PraqParameters p = *parameters;
    if (!praq::valid(p)) return PRAQ_ERROR_ARGUMENT;
    praq::HostLayout L;
    const int st = praq::build_layout(*instance, L);
    if (st) return st;
    if (p.max_iter <= 0) p.max_iter = -1;
    if (p.op_steps <= 0) p.op_steps = praq_check_interval(instance->n, &p);
    if (p.op_steps < 2) p.op_steps = 2;
    auto solver = std::make_unique<reform_praq_solver>();
    auto make = [&](auto* impl) -> int {
        impl->L = std::move(L);
        impl->p = p;
        solver->impl.reset(impl);
        return impl->setup(static_cast<cudaStream_t>(stream)) == cudaSuccess ? 0 : PRAQ_ERROR_CUDA;
    };
    const int rc = p.use_float32 ? make(new praq::Solver<float>()) : make(new praq::Solver<double>());
    if (rc) return rc;
    *out = solver.release();
    return 0;
}

int reform_praq_run(reform_praq_solver* solver) {
    if (!solver || !solver->impl) return PRAQ_ERROR_ARGUMENT;
    return solver->impl->run();
}

int reform_praq_result(reform_praq_solver* solver, double* x, double* y2, PraqResult* result) {
    if (!solver || !solver->impl) return PRAQ_ERROR_ARGUMENT;
    return solver->impl->result(x, y2, result);
}

int reform_praq_set_time_limit(reform_praq_solver* solver, double seconds) {
    if (!solver || !solver->impl) return PRAQ_ERROR_ARGUMENT;
    solver->impl->time_limit = seconds;
    return 0;
}

int reform_praq_run_profiled(reform_praq_solver* solver, double* ms, int64_t* count) {
    if (!solver || !solver->impl || !ms || !count) return PRAQ_ERROR_ARGUMENT;
    long long c[9];
    const int st = solver->impl->run_profiled(ms, c);
    for (int k = 0; k < 9; ++k) count[k] = c[k];
    return st;
}

int64_t reform_praq_launches(const reform_praq_solver* solver) {
    return solver && solver->impl ? solver->impl->launches() : 0;
}

void reform_praq_destroy(reform_praq_solver* solver) { delete solver; }

int praq_solve(const PraqInstance* instance, const PraqParameters* parameters, double* x,
               PraqResult* result) {
    if (result) {
        result->lower = std::numeric_limits<double>::quiet_NaN();
        result->upper = std::numeric_limits<double>::quiet_NaN();
        result->iterations = 0;
        result->status = PRAQ_ERROR_ARGUMENT;
    }
    if (!instance || !parameters || !x || !result) return PRAQ_ERROR_ARGUMENT;
    reform_praq_solver* s = nullptr;
    int st = reform_praq_create(instance, parameters, nullptr, &s);
    if (st) {
        result->status = st;
        return st;
    }
    st = reform_praq_run(s);
    if (st >= 0) {
        const int rs = reform_praq_result(s, x, nullptr, result);
        if (rs) st = rs;
    }
    reform_praq_destroy(s);
    if (st < 0) result->status = st;
    return st;
}

}  // extern "C"
