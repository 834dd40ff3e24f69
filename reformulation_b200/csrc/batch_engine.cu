// batch_engine.cu -- many PRAQ and PRIA instances of uneven size in one engine
// (include/reform.h).
//
// Each instance keeps the device layout and iterates of its solo solver
// (praq_core.cuh, pria_core.cuh); this file is a second driver over them.  Per
// kernel kind there is ONE launch covering every active instance: the work is
// listed in device-resident tables of (instance, tile) pairs, and a persistent
// grid (a fixed number of CTAs per SM, or of clusters for the JRP y/z
// half-step, grouped by cluster size) walks the table.  Each tile runs the
// same tile function as the solo kernel, with the instance's descriptor
// copied into shared memory, so every instance computes bitwise what its solo
// solve computes.  Per-instance restart and termination state stays on the
// device (each instance's control block); one op_steps block of all
// instances -- steps, bounds, checks, the gated restart steps, a gather of
// all control blocks into one host copy -- is one captured CUDA graph.
// Between replays the host retires finished instances by rewriting the tables
// and their counts (device memory the graph reads), so the graph is replayed
// unchanged; instances can also join between replays.
#include "../../include/reform.h"
#include "praq_core.cuh"
#include "pria_core.cuh"

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <tuple>
#include <vector>

namespace rb200 {
namespace batch {
namespace {

struct QMeta {
    praq::Params prm;
    int nbn, nbe;
};
struct JMeta {
    pria::Params prm;
    int nbx, nby, nbyz, nbup, nblo;
};

// One instance's state as the host needs it after a block.
struct Summary {
    double lower, upper, gap;
    long long iteration;
    int terminated, restart;
};

// JRP x tiles fall into classes by the shared memory they need (their row
// count), each class launched with its own dynamic shared memory, so that the
// longest horizon in the batch does not set every tile's occupancy.
constexpr int kXClasses = 4;
constexpr int kXClassRows[kXClasses] = {127, 255, 511, pria::kMaxPeriods + 1};   // rows | 1 at most

enum Count { kNode = 0, kEdge, kQLow, kUp, kJLow, kQCheck, kJCheck, kY, kX0 };
constexpr int kYZ0 = kX0 + kXClasses;
constexpr int kMaxGroups = 17;   // y/z cluster sizes 1..16
// JRPs of at least this many packed entries run their step kernels as their
// own launches (the solo solver's grids, one instance after the other on one
// branch of the graph); the smaller ones share the table-driven persistent
// kernels.
constexpr long long kBigJrp = 1LL << 20;
constexpr size_t kBigStream0 = 32;   // the auxiliary stream of the big JRPs' chain
constexpr int kCounts = kYZ0 + kMaxGroups;

// --- batched kernels: persistent grids over the work tables ---------------

// The persistent grids walk their table (task t, t + stride, ...) with the
// next task's instance descriptor fetched into the second of two shared
// slots by cp.async while the current task runs, so no task waits on its
// descriptor's load: body(descriptor in shared memory, task).
template <class D>
__device__ __forceinline__ void desc_fetch(D* dst, const D* src) {
    static_assert(sizeof(D) % 16 == 0 && alignof(D) >= 16, "descriptors move in 16-byte pieces");
    constexpr int kPieces = int(sizeof(D) / 16);
    if (int(threadIdx.x) < kPieces) {
        const unsigned s = unsigned(__cvta_generic_to_shared(reinterpret_cast<char*>(dst) + 16 * threadIdx.x));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s),
                     "l"(reinterpret_cast<const char*>(src) + 16 * threadIdx.x)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

template <class D, class Body>
__device__ __forceinline__ void walk_tasks(const D* devs, const int2* tasks, int total, int first, int stride,
                                           D (&slot)[2], Body body) {
    if (first >= total) return;
    int2 w = tasks[first];
    desc_fetch(&slot[0], devs + w.x);
    int b = 0;
    for (int t = first; t < total; t += stride, b ^= 1) {
        const int2 cur = w;
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();   // slot b complete for every thread; every thread done with slot b ^ 1
        if (t + stride < total) {
            w = tasks[t + stride];
            desc_fetch(&slot[b ^ 1], devs + w.x);
        }
        body(slot[b], cur);
    }
}

template <class Real, bool Reflect, bool Check>
__global__ void __launch_bounds__(praq::kBlock)
bq_node(const praq::Dev<Real>* devs, const int2* __restrict__ tiles, const int* count, int step, int gate) {
    __shared__ praq::Dev<Real> slot[2];
    walk_tasks(devs, tiles, *count, int(blockIdx.x), int(gridDim.x), slot, [&](const praq::Dev<Real>& sd, int2 w) {
        praq::node_kernel_tile<Real, Reflect, Check>(sd, w.y, Reflect ? sd.pred : sd.u2s,
                                                     Reflect ? sd.pred1 : sd.u2s1, step, 0, gate);
    });
}

template <class Real, bool Reflect, bool Check>
__global__ void __launch_bounds__(praq::kBlock)
bq_edge(const praq::Dev<Real>* devs, const int2* __restrict__ tiles, const int* count, int step, int gate) {
    __shared__ praq::Dev<Real> slot[2];
    walk_tasks(devs, tiles, *count, int(blockIdx.x), int(gridDim.x), slot, [&](const praq::Dev<Real>& sd, int2 w) {
        praq::edge_kernel_tile<Real, Reflect, Check>(sd, w.y, Reflect ? nullptr : sd.u2s, step, 0, gate);
    });
}

template <class Real>
__global__ void __launch_bounds__(praq::kBlock)
bq_lower(const praq::Dev<Real>* devs, const int2* __restrict__ tiles, const int* count) {
    __shared__ praq::Dev<Real> slot[2];
    walk_tasks(devs, tiles, *count, int(blockIdx.x), int(gridDim.x), slot, [&](const praq::Dev<Real>& sd, int2 w) {
        praq::lower_kernel_tile<Real>(sd, w.y, sd.u2s, sd.u2s1);
    });
}

template <class Real>
__global__ void __launch_bounds__(praq::kCheckBlock)
bq_check(const praq::Dev<Real>* devs, const QMeta* metas, const int* __restrict__ list, const int* count,
         int mode) {
    const int total = *count;
    for (int k = blockIdx.x; k < total; k += gridDim.x) {
        const int id = list[k];
        const praq::Dev<Real>& d = devs[id];
        const QMeta& m = metas[id];
        praq::check_body(d.ctl, m.prm, d.scale, d.pnode, m.nbn, d.pedge, m.nbe, d.plower, m.nbn, mode);
        __syncthreads();
    }
}

template <class Real, int TW, bool Reflect, bool Check>
__global__ void __launch_bounds__(pria::kXThreads)
bj_x(const pria::Dev<Real>* devs, const int2* __restrict__ tiles, const int* count, int step, int gate) {
    __shared__ pria::Dev<Real> slot[2];
    walk_tasks(devs, tiles, *count, int(blockIdx.x), int(gridDim.x), slot, [&](const pria::Dev<Real>& sd, int2 w) {
        if (Reflect)
            pria::x_kernel_tile<Real, TW, Reflect, Check>(sd, w.y, sd.xh, sd.yh, sd.zh, step, gate);
        else
            pria::x_kernel_tile<Real, TW, Reflect, Check>(sd, w.y, sd.x2s, sd.y2s, sd.z2s, step, gate);
    });
}

template <class Real, bool Reflect, bool Check>
__global__ void __launch_bounds__(pria::kYThreads)
bj_y(const pria::Dev<Real>* devs, const int2* __restrict__ tiles, const int* count, int step, int gate) {
    __shared__ pria::Dev<Real> slot[2];
    extern __shared__ __align__(16) unsigned char smem_raw[];   // kYThreads / 32 rows of kMaxPeriods
    walk_tasks(devs, tiles, *count, int(blockIdx.x), int(gridDim.x), slot, [&](const pria::Dev<Real>& sd, int2 w) {
        pria::y_kernel_tile<Real, Reflect, Check>(sd, w.y, Reflect ? sd.yh : sd.y2s, step, gate,
                                                  reinterpret_cast<Real*>(smem_raw), pria::kMaxPeriods);
    });
}

// Persistent clusters: cluster c takes tasks c, c + clusters, ...; every CTA
// of a cluster takes the same task (the z half-step of one period block).
template <class Real, int kThreads, bool Reflect, bool Check>
__global__ void __launch_bounds__(kThreads)
bj_z(const pria::Dev<Real>* devs, const int2* __restrict__ tasks, const int* count, int csize, int step,
     int gate) {
    __shared__ pria::Dev<Real> slot[2];
    const int nclusters = int(gridDim.x) / csize;
    walk_tasks(devs, tasks, *count, int(blockIdx.x) / csize, nclusters, slot, [&](const pria::Dev<Real>& sd, int2 w) {
        pria::z_task<Real, kThreads, Reflect, Check>(sd, w.y, Reflect ? sd.zh : sd.z2s, step, gate);
    });
}

template <class Real>
__global__ void __launch_bounds__(pria::kAuxThreads)
bj_upper(const pria::Dev<Real>* devs, const int2* __restrict__ tasks, const int* count) {
    __shared__ pria::Dev<Real> slot[2];
    walk_tasks(devs, tasks, *count, int(blockIdx.x), int(gridDim.x), slot, [&](const pria::Dev<Real>& sd, int2 w) {
        pria::upper_kernel_tile<Real>(sd, w.y, sd.x2s, sd.tp, 0);
    });
}

template <class Real>
__global__ void __launch_bounds__(pria::kAuxThreads)
bj_lower(const pria::Dev<Real>* devs, const int2* __restrict__ tiles, const int* count) {
    __shared__ pria::Dev<Real> slot[2];
    walk_tasks(devs, tiles, *count, int(blockIdx.x), int(gridDim.x), slot, [&](const pria::Dev<Real>& sd, int2 w) {
        pria::lower_kernel_tile<Real>(sd, w.y, sd.y2s, sd.z2s);
    });
}

template <class Real>
__global__ void __launch_bounds__(pria::kCheckBlock)
bj_check(const pria::Dev<Real>* devs, const JMeta* metas, const int* __restrict__ list, const int* count,
         int mode) {
    const int total = *count;
    for (int k = blockIdx.x; k < total; k += gridDim.x) {
        const int id = list[k];
        const pria::Dev<Real>& d = devs[id];
        const JMeta& m = metas[id];
        pria::check_body(d.ctl, m.prm, d.px, m.nbx, d.py, m.nby, d.pyz, m.nbyz, d.pup, m.nbup, d.plo, m.nblo, mode);
        __syncthreads();
    }
}

// Every running instance's control block into one array, at the instance's
// id (ids are never reused, so a block captured before instances joined
// still writes every instance it covers to the right place).
template <class Real>
__global__ void b_gather(const praq::Dev<Real>* qdevs, const int* __restrict__ qid, int nq,
                         const pria::Dev<Real>* jdevs, const int* __restrict__ jid, int nj,
                         const unsigned char* __restrict__ live, Summary* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nq + nj) return;
    const int id = k < nq ? qid[k] : jid[k - nq];
    if (!live[id]) return;
    Summary s;
    if (k < nq) {
        const praq::Control* c = qdevs[k].ctl;
        s = Summary{c->lower, c->upper, c->gap, c->iteration, c->terminated, c->restart};
    } else {
        const pria::Control* c = jdevs[k - nq].ctl;
        s = Summary{c->lower, c->upper, c->gap, c->iteration, c->terminated, c->restart};
    }
    out[id] = s;
}

template <class T>
struct Table {
    PoolBuf<T> buf;
    std::vector<T> host;
    size_t capacity = 0;
};

struct Shapes {
    int grid_mult = 8;
};

std::mutex tuned_mu;
std::map<std::tuple<int, int, int, int, int>, Shapes> tuned;   // size class -> shapes

struct EngineBase {
    virtual ~EngineBase() = default;
    virtual int add_qubo(const PraqInstance& in, const PraqParameters& p) = 0;
    virtual int add_jrp(int64_t n, int64_t t, const double* k, double k0, const double* h,
                        const pria_params& p) = 0;
    virtual int add_jrp_demand(int64_t n, int64_t t, const double* k, double k0, const double* rate,
                               const double* demand, const pria_params& p) = 0;
    virtual int start() = 0;
    virtual int run(int64_t max_blocks) = 0;
    virtual int launch() = 0;
    virtual int sync(int* ids, int max, int* count) = 0;
    virtual int inflight() const = 0;
    virtual int status(int id, int* done, int64_t* it, double* lo, double* up) = 0;
    virtual int result_qubo(int id, double* x, PraqResult* r) = 0;
    virtual int set_warm_qubo(int id, const double* x, const double* y2) = 0;
    virtual int point_qubo(int id, double* x, double* y2) = 0;
    virtual int result_jrp(int id, double* x, double* y, double* z, pria_result_info* info) = 0;
    virtual int remove(int id) = 0;
    virtual int64_t device_bytes() const = 0;
    virtual int set_shapes(const reform_shapes& s) = 0;
    virtual int autotune(reform_shapes* out) = 0;
    virtual int64_t launches() const = 0;
    virtual int restart() = 0;
};

template <class Real>
struct Engine final : EngineBase {
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // Instances are laid out on their own stream, so that a layout (uploads,
    // sorts, packing) overlaps the blocks already queued on `stream`; the
    // engine's stream then waits for it before the instance is started.
    cudaStream_t lay = nullptr;
    cudaEvent_t lay_done = nullptr;
    int sms = 148;
    int op_steps = 0;
    Shapes shapes;
    bool shapes_fixed = false;

    struct QInst {
        std::unique_ptr<praq::Solver<Real>> s;
        bool started = false, done = false, live = true;
        Summary last{};
        long long join = 0;   // the first block that includes it
    };
    struct JInst {
        std::unique_ptr<pria::Solver<Real>> s;
        bool started = false, done = false, live = true;
        Summary last{};
        long long join = 0;
    };
    long long launched = 0, synced = 0;   // blocks enqueued / inspected so far
    std::vector<QInst> q;
    std::vector<JInst> j;
    std::vector<std::pair<int, int>> ids;   // id -> (0 QUBO / 1 JRP, index)

    // device copies of descriptors and meta (indexed by instance slot)
    Table<praq::Dev<Real>> qdevs;
    Table<QMeta> qmeta;
    Table<pria::Dev<Real>> jdevs;
    Table<JMeta> jmeta;
    Table<int2> t_node, t_edge, t_qlow, t_up, t_jlow, t_y;
    Table<int2> t_x[kXClasses];
    Table<int2> t_yz[kMaxGroups];
    Table<int> l_qcheck, l_jcheck;
    Table<int> qid_t, jid_t;          // QUBO / JRP index -> id
    Table<unsigned char> live;        // per id: running in the current tables
    PoolBuf<int> counts;
    PoolBuf<Summary> summary;
    Summary* hsummary = nullptr;
    size_t hsummary_cap = 0;
    int hcounts[kCounts] = {};

    size_t yz_smem[kMaxGroups] = {};
    bool groups[kMaxGroups] = {};
    bool xclasses[kXClasses] = {};
    bool graph_q = false, graph_j = false;   // the captured block has QUBO / JRP work
    std::vector<int> jbig;                    // running big JRPs in the captured block
    static constexpr int tw = pria::kXTile;
    bool dirty = true;          // the graph must be captured again
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaEvent_t> events;
    int head = 0, pending = 0;   // ring of enqueued blocks
    long long nlaunch = 0, block_nodes = 0;

    ~Engine() override {
        if (stream) cudaStreamSynchronize(stream);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto ev : events) cudaEventDestroy(ev);
        for (auto ev : fj) cudaEventDestroy(ev);
        for (auto st : aux) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        q.clear();
        j.clear();
        graves.clear();
        if (lay) {   // the instances' buffers were freed on the layout stream
            cudaStreamSynchronize(lay);
            cudaStreamDestroy(lay);
        }
        if (lay_done) cudaEventDestroy(lay_done);
        // every stream-ordered free before the stream goes away
        qdevs.buf.release();
        qmeta.buf.release();
        jdevs.buf.release();
        jmeta.buf.release();
        for (auto* tb : {&t_node, &t_edge, &t_qlow, &t_up, &t_jlow, &t_y}) tb->buf.release();
        for (auto& tb : t_x) tb.buf.release();
        for (auto& tb : t_yz) tb.buf.release();
        l_qcheck.buf.release();
        l_jcheck.buf.release();
        qid_t.buf.release();
        jid_t.buf.release();
        live.buf.release();
        counts.release();
        summary.release();
        if (stream) cudaStreamSynchronize(stream);
        if (hsummary) cudaFreeHost(hsummary);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    int init(cudaStream_t s) {
        (void)cudaGetLastError();   // a stale error of an unrelated earlier call is not ours
        if (s) {
            stream = s;
        } else {
            if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)) return -int(cudaErrorUnknown);
            own_stream = true;
        }
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaStreamCreateWithFlags(&lay, cudaStreamNonBlocking) ||
            cudaEventCreateWithFlags(&lay_done, cudaEventDisableTiming))
            return -int(cudaErrorUnknown);
        if (counts.alloc(kCounts, stream)) return -int(cudaErrorMemoryAllocation);
        events.resize(4);
        for (auto& ev : events)
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) return -int(cudaErrorUnknown);
        return 0;
    }

    int add_qubo(const PraqInstance& in, const PraqParameters& p0) override {
        PraqParameters p = p0;
        if (!praq::valid(p)) return PRAQ_ERROR_ARGUMENT;
        if (p.max_iter <= 0) p.max_iter = -1;
        if (op_steps == 0) op_steps = int(p.op_steps > 0 ? std::max<int64_t>(p.op_steps, 2) : 16);
        p.op_steps = op_steps;
        auto s = std::make_unique<praq::Solver<Real>>();
        s->p = p;
        s->allow_pull = false;   // the engine's kernels read slot 1 in the push layout
        s->allow_mega = false;   // the engine runs its own kernels
        const int st = s->setup(in, lay);
        if (st) return st;
        if (joined(s->stream)) return PRAQ_ERROR_CUDA;
        q.push_back(QInst{std::move(s)});
        ids.emplace_back(0, int(q.size()) - 1);
        dirty = true;
        return int(ids.size()) - 1;
    }

    int add_jrp(int64_t n, int64_t t, const double* k, double k0, const double* h,
                const pria_params& p0) override {
        pria_params p = p0;
        if (!p.use_halpern || p.warm_steps > 0) return -int(cudaErrorNotSupported);   // Halpern blocks only
        if (op_steps == 0) op_steps = std::max(p.op_steps, 2);
        p.op_steps = op_steps;
        std::unique_ptr<pria::SolverBase> base;
        const int st = pria::create<double>(n, t, k, k0, h, &p, sizeof(Real) == 4, lay, base);
        if (st) return -st;
        std::unique_ptr<pria::Solver<Real>> s(static_cast<pria::Solver<Real>*>(base.release()));
        if (joined(s->stream)) return -int(cudaErrorUnknown);
        j.push_back(JInst{std::move(s)});
        ids.emplace_back(1, int(j.size()) - 1);
        dirty = true;
        return int(ids.size()) - 1;
    }

    int add_jrp_demand(int64_t n, int64_t t, const double* k, double k0, const double* rate, const double* demand,
                       const pria_params& p0) override {
        pria_params p = p0;
        if (!p.use_halpern || p.warm_steps > 0) return -int(cudaErrorNotSupported);   // Halpern blocks only
        if (op_steps == 0) op_steps = std::max(p.op_steps, 2);
        p.op_steps = op_steps;
        std::unique_ptr<pria::SolverBase> base;
        const int st = pria::create_demand(n, t, k, k0, rate, demand, &p, sizeof(Real) == 4, lay, base);
        if (st) return -st;
        std::unique_ptr<pria::Solver<Real>> s(static_cast<pria::Solver<Real>*>(base.release()));
        if (joined(s->stream)) return -int(cudaErrorUnknown);
        j.push_back(JInst{std::move(s)});
        ids.emplace_back(1, int(j.size()) - 1);
        dirty = true;
        return int(ids.size()) - 1;
    }

    // A freshly laid-out instance joins the engine's stream: the stream waits
    // for its layout, and every later operation of the instance (its start,
    // result reads, warm starts) is ordered on the engine's stream.  Its
    // buffers keep freeing on the layout stream, which happens only after the
    // engine's stream has been drained (remove, destruction).
    int joined(cudaStream_t& solver_stream) {
        if (cudaEventRecord(lay_done, lay) || cudaStreamWaitEvent(stream, lay_done, 0)) return 1;
        solver_stream = stream;
        return 0;
    }

    template <class T>
    int upload(Table<T>& tb) {
        if (tb.host.size() > tb.capacity) {
            tb.capacity = std::max<size_t>(tb.host.size() * 2, 64);
            if (tb.buf.alloc(tb.capacity, stream)) return -int(cudaErrorMemoryAllocation);
            dirty = true;
        }
        if (!tb.host.empty() &&
            cudaMemcpyAsync(tb.buf.ptr, tb.host.data(), sizeof(T) * tb.host.size(), cudaMemcpyHostToDevice,
                            stream))
            return -int(cudaErrorUnknown);
        return 0;
    }

    // The work tables of the instances that are started and not done,
    // heaviest tiles first within each kind.
    int rebuild() {
        qdevs.host.clear();
        qmeta.host.clear();
        for (auto& qi : q) {
            qdevs.host.push_back(qi.s ? qi.s->d : praq::Dev<Real>{});
            QMeta m{};
            if (qi.s) m = QMeta{qi.s->prm, qi.s->nb_node, qi.s->nb_edge};
            qmeta.host.push_back(m);
        }
        jdevs.host.clear();
        jmeta.host.clear();
        for (auto& ji : j) {
            jdevs.host.push_back(ji.s ? ji.s->d : pria::Dev<Real>{});
            JMeta m{};
            if (ji.s) m = JMeta{ji.s->prm, ji.s->nbx, ji.s->nby, ji.s->nbyz, ji.s->tp, ji.s->nblo};
            jmeta.host.push_back(m);
        }
        for (auto* tb : {&t_node, &t_edge, &t_qlow, &t_up, &t_jlow, &t_y}) tb->host.clear();
        for (auto& tb : t_x) tb.host.clear();
        for (auto& tb : t_yz) tb.host.clear();
        l_qcheck.host.clear();
        l_jcheck.host.clear();
        live.host.assign(ids.size(), 0);
        qid_t.host.assign(q.size(), 0);
        jid_t.host.assign(j.size(), 0);
        for (int id = 0; id < int(ids.size()); ++id)
            (ids[id].first == 0 ? qid_t.host[ids[id].second] : jid_t.host[ids[id].second]) = id;
        size_t ys[kMaxGroups] = {};
        bool gr[kMaxGroups] = {};
        for (int k = 0; k < int(q.size()); ++k) {
            auto& qi = q[k];
            if (!qi.s || !qi.started || qi.done) continue;
            live.host[qid_t.host[k]] = 1;
            for (int t = 0; t < qi.s->nb_node; ++t) {
                t_node.host.push_back(make_int2(k, t));
                t_qlow.host.push_back(make_int2(k, t));
            }
            if (qi.s->m)
                for (int t = 0; t < qi.s->nb_edge; ++t) t_edge.host.push_back(make_int2(k, t));
            l_qcheck.host.push_back(k);
        }
        // JRP: x tiles sorted by rows (cost), y/z tasks by block size
        std::vector<std::pair<long long, int2>> xt[kXClasses], yzt[kMaxGroups], upt, yt;
        std::vector<int> big_now;
        for (int k = 0; k < int(j.size()); ++k) {
            auto& ji = j[k];
            if (!ji.s || !ji.started || ji.done) continue;
            live.host[jid_t.host[k]] = 1;
            auto& s = *ji.s;
            const int n = s.n, tp = s.tp, ntc = s.d.ntc;
            const bool big = s.nd >= kBigJrp;
            if (big) big_now.push_back(k);
            for (int t = 0; !big && t < n * ntc; ++t) {
                const int ctile = ntc - 1 - t / n;
                const int rows = std::min(tp, (ctile + 1) * s.tw);
                int cls = 0;
                while ((rows | 1) > kXClassRows[cls]) ++cls;
                xt[cls].emplace_back((long long)rows, make_int2(k, t));
            }
            const int c = s.d.csize;
            if (!big) {
                gr[c] = true;
                ys[c] = std::max(ys[c], s.yz_smem);
            }
            for (int sb = 0; sb < tp; ++sb) {
                if (!big) yzt[c].emplace_back((long long)n * (tp - sb), make_int2(k, sb));
                upt.emplace_back((long long)n * (tp - sb), make_int2(k, sb));
            }
            for (int t = 0; t < s.nblo; ++t) t_jlow.host.push_back(make_int2(k, t));
            for (int t = 0; !big && t < s.nby; ++t) {
                const long long row = (long long)t * (pria::kYThreads / 32);
                yt.emplace_back((long long)(tp - int(row / n)), make_int2(k, t));   // row length
            }
            l_jcheck.host.push_back(k);
        }
        auto order = [](std::vector<std::pair<long long, int2>>& v, Table<int2>& out) {
            std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
            for (auto& e : v) out.host.push_back(e.second);
        };
        const bool run_q = !l_qcheck.host.empty(), run_j = !l_jcheck.host.empty();
        if (big_now != jbig) {
            jbig = big_now;
            dirty = true;
        }
        if (run_q != graph_q || run_j != graph_j) {
            graph_q = run_q;
            graph_j = run_j;
            dirty = true;
        }
        for (int c = 0; c < kXClasses; ++c) {
            order(xt[c], t_x[c]);
            if (!xt[c].empty() && !xclasses[c]) {
                xclasses[c] = true;
                dirty = true;
            }
        }
        order(upt, t_up);
        order(yt, t_y);
        for (int c = 1; c < kMaxGroups; ++c) order(yzt[c], t_yz[c]);
        for (int c = 1; c < kMaxGroups; ++c) {
            if (gr[c] && (!groups[c] || ys[c] > yz_smem[c])) dirty = true;
            if (gr[c]) {
                groups[c] = true;
                yz_smem[c] = std::max(yz_smem[c], ys[c]);
            }
        }
        int rc = 0;
        if ((rc = upload(qdevs)) || (rc = upload(qmeta)) || (rc = upload(jdevs)) || (rc = upload(jmeta))) return rc;
        for (auto* tb : {&t_node, &t_edge, &t_qlow, &t_up, &t_jlow, &t_y})
            if ((rc = upload(*tb))) return rc;
        for (int c = 0; c < kXClasses; ++c)
            if (xclasses[c] && (rc = upload(t_x[c]))) return rc;
        for (int c = 1; c < kMaxGroups; ++c)
            if (groups[c] && (rc = upload(t_yz[c]))) return rc;
        if ((rc = upload(l_qcheck)) || (rc = upload(l_jcheck)) || (rc = upload(live)) || (rc = upload(qid_t)) ||
            (rc = upload(jid_t)))
            return rc;
        hcounts[kNode] = int(t_node.host.size());
        hcounts[kEdge] = int(t_edge.host.size());
        hcounts[kQLow] = int(t_qlow.host.size());
        for (int c = 0; c < kXClasses; ++c) hcounts[kX0 + c] = int(t_x[c].host.size());
        hcounts[kUp] = int(t_up.host.size());
        hcounts[kJLow] = int(t_jlow.host.size());
        hcounts[kY] = int(t_y.host.size());
        hcounts[kQCheck] = int(l_qcheck.host.size());
        hcounts[kJCheck] = int(l_jcheck.host.size());
        for (int c = 0; c < kMaxGroups; ++c) hcounts[kYZ0 + c] = int(t_yz[c].host.size());
        if (cudaMemcpyAsync(counts.ptr, hcounts, sizeof(hcounts), cudaMemcpyHostToDevice, stream))
            return -int(cudaErrorUnknown);
        const size_t slots = ids.size();
        if (summary.count < slots) {
            if (summary.alloc(std::max<size_t>(slots * 2, 64), stream)) return -int(cudaErrorMemoryAllocation);
            dirty = true;
        }
        if (hsummary_cap < summary.count) {
            if (pending && drain()) return -int(cudaErrorUnknown);   // a block may still copy into it
            if (hsummary) cudaFreeHost(hsummary);
            hsummary = nullptr;
            if (cudaMallocHost(reinterpret_cast<void**>(&hsummary), sizeof(Summary) * summary.count))
                return -int(cudaErrorMemoryAllocation);
            std::memset(hsummary, 0, sizeof(Summary) * summary.count);
            hsummary_cap = summary.count;
        }
        // (host-to-device copies from pageable memory are staged when issued)
        return 0;
    }

    static constexpr size_t x_class_smem(int c) { return size_t(tw) * size_t(kXClassRows[c]) * sizeof(double); }

    template <bool R, bool C>
    cudaError_t launch_x(int c, int step, int gate, cudaStream_t st) {
        const size_t smem = x_class_smem(c);
        const int per_sm = std::max(1, std::min(8, int((228 * 1024) / (smem + 2048))));
        bj_x<Real, tw, R, C><<<sms * per_sm, pria::kXThreads, smem, st>>>(jdevs.buf.ptr, t_x[c].buf.ptr,
                                                                         counts.ptr + kX0 + c, step, gate);
        return cudaGetLastError();
    }

    template <bool R, bool C>
    cudaError_t launch_y(int step, int gate, cudaStream_t st) {
        const size_t smem = pria::Solver<Real>::y_smem_limit();
        bj_y<Real, R, C><<<sms * std::max(1, int((228 * 1024) / (smem + 2048))), pria::kYThreads, smem, st>>>(
            jdevs.buf.ptr, t_y.buf.ptr, counts.ptr + kY, step, gate);
        return cudaGetLastError();
    }

    template <bool R, bool C>
    cudaError_t launch_yz(int c, int step, int gate, cudaStream_t st) {
        constexpr int kT = pria::z_threads<Real>();
        const int per_sm = std::max(1, int((228 * 1024) / (yz_smem[c] + 4096)));
        const int nclusters = std::max(1, (sms * std::min(per_sm, 2)) / c);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(unsigned(nclusters * c));
        cfg.blockDim = dim3(kT);
        cfg.dynamicSmemBytes = yz_smem[c];
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = unsigned(c);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, bj_z<Real, kT, R, C>, (const pria::Dev<Real>*)jdevs.buf.ptr,
                                  (const int2*)t_yz[c].buf.ptr, (const int*)(counts.ptr + kYZ0 + c), c, step,
                                  gate);
    }

    // Limits at the most any instance can ask for, not this engine's current
    // need: the attribute belongs to the kernel and is shared by every engine
    // in the process (the same rule as the single-instance solver's).
    cudaError_t set_attributes() {
        const size_t xlim = pria::Solver<Real>::x_smem_limit();
        static_assert(x_class_smem(kXClasses - 1) <= pria::Solver<Real>::x_smem_limit(), "x class fits");
        auto xa = [&](auto fn) {
            return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(xlim));
        };
        RB_CUDA_TRY(xa(bj_x<Real, tw, true, false>));
        RB_CUDA_TRY(xa(bj_x<Real, tw, true, true>));
        RB_CUDA_TRY(xa(bj_x<Real, tw, false, true>));
        auto yattr = [&](auto fn) {
            return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(pria::Solver<Real>::y_smem_limit()));
        };
        RB_CUDA_TRY(yattr(bj_y<Real, true, false>));
        RB_CUDA_TRY(yattr(bj_y<Real, true, true>));
        RB_CUDA_TRY(yattr(bj_y<Real, false, true>));
        constexpr int kT = pria::z_threads<Real>();
        auto ya = [&](auto fn) -> cudaError_t {
            RB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, pria::z_slice_bytes<Real>()));
            return cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        };
        RB_CUDA_TRY(ya(bj_z<Real, kT, true, false>));
        RB_CUDA_TRY(ya(bj_z<Real, kT, true, true>));
        RB_CUDA_TRY(ya(bj_z<Real, kT, false, true>));
        return cudaSuccess;
    }

    // --- fork/join on auxiliary streams (graph branches under capture) -----
    std::vector<cudaStream_t> aux;
    std::vector<cudaEvent_t> fj;
    size_t fj_next = 0;

    cudaError_t aux_stream(size_t k, cudaStream_t* out) {
        while (aux.size() <= k) {
            cudaStream_t st;
            RB_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            aux.push_back(st);
        }
        *out = aux[k];
        return cudaSuccess;
    }
    // `to` waits for everything enqueued on `from` so far
    cudaError_t order_after(cudaStream_t from, cudaStream_t to) {
        if (fj_next == fj.size()) {
            cudaEvent_t ev;
            RB_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            fj.push_back(ev);
        }
        cudaEvent_t ev = fj[fj_next++];
        RB_CUDA_TRY(cudaEventRecord(ev, from));
        return cudaStreamWaitEvent(to, ev, 0);
    }

    // One op_steps block of every instance.  The QUBO steps and the JRP steps
    // are independent chains (separate branches of the graph), and within a
    // JRP half-step the x shared-memory classes and the y/z cluster-size
    // groups run side by side; the gather of all control blocks joins them.
    cudaError_t enqueue_block() {
        const int gq = sms * shapes.grid_mult;
        // only the kinds with running instances (a retired kind leaves the graph)
        const bool hq = graph_q, hj = graph_j;
        long long nodes = 0;
        fj_next = 0;
        cudaStream_t sq = stream;
        if (hq && hj) {
            RB_CUDA_TRY(aux_stream(0, &sq));
            RB_CUDA_TRY(order_after(stream, sq));
        }
        if (hq) {
            for (int s = 0; s < op_steps; ++s) {
                if (s + 1 == op_steps) {
                    bq_node<Real, true, true><<<gq, praq::kBlock, 0, sq>>>(qdevs.buf.ptr, t_node.buf.ptr, counts.ptr + kNode, s, 0);
                    bq_edge<Real, true, true><<<gq, praq::kBlock, 0, sq>>>(qdevs.buf.ptr, t_edge.buf.ptr, counts.ptr + kEdge, s, 0);
                } else {
                    bq_node<Real, true, false><<<gq, praq::kBlock, 0, sq>>>(qdevs.buf.ptr, t_node.buf.ptr, counts.ptr + kNode, s, 0);
                    bq_edge<Real, true, false><<<gq, praq::kBlock, 0, sq>>>(qdevs.buf.ptr, t_edge.buf.ptr, counts.ptr + kEdge, s, 0);
                }
                nodes += 2;
            }
            bq_lower<Real><<<gq, praq::kBlock, 0, sq>>>(qdevs.buf.ptr, t_qlow.buf.ptr, counts.ptr + kQLow);
            bq_check<Real><<<sms * 4, praq::kCheckBlock, 0, sq>>>(qdevs.buf.ptr, qmeta.buf.ptr, l_qcheck.buf.ptr,
                                                                 counts.ptr + kQCheck, 1);
            bq_node<Real, false, true><<<gq, praq::kBlock, 0, sq>>>(qdevs.buf.ptr, t_node.buf.ptr, counts.ptr + kNode, 0, 1);
            bq_edge<Real, false, true><<<gq, praq::kBlock, 0, sq>>>(qdevs.buf.ptr, t_edge.buf.ptr, counts.ptr + kEdge, 0, 1);
            bq_check<Real><<<sms * 4, praq::kCheckBlock, 0, sq>>>(qdevs.buf.ptr, qmeta.buf.ptr, l_qcheck.buf.ptr,
                                                                 counts.ptr + kQCheck, 2);
            nodes += 5;
        }
        if (hj) {
            // the x classes of one half-step, side by side
            auto x_stage = [&](auto launch_one) -> cudaError_t {
                size_t k = 1;
                bool first = true;
                for (int c = 0; c < kXClasses; ++c) {
                    if (!xclasses[c]) continue;
                    cudaStream_t st = stream;
                    if (!first) {
                        RB_CUDA_TRY(aux_stream(k++, &st));
                        RB_CUDA_TRY(order_after(stream, st));
                    }
                    RB_CUDA_TRY(launch_one(c, st));
                    ++nodes;
                    first = false;
                }
                for (size_t a = 1; a < k; ++a) RB_CUDA_TRY(order_after(aux[a], stream));
                return cudaSuccess;
            };
            // the y half-step beside the z cluster-size groups
            auto yz_stage = [&](auto launch_y_one, auto launch_one) -> cudaError_t {
                size_t k = 1;
                int zgroup[kMaxGroups];
                int nz = 0;
                for (int c = 1; c < kMaxGroups; ++c) {   // fork every z group off the main stream first
                    if (!groups[c]) continue;
                    cudaStream_t st;
                    RB_CUDA_TRY(aux_stream(k++, &st));
                    RB_CUDA_TRY(order_after(stream, st));
                    zgroup[nz++] = c;
                }
                RB_CUDA_TRY(launch_y_one(stream));
                ++nodes;
                for (int g = 0; g < nz; ++g) {
                    RB_CUDA_TRY(launch_one(zgroup[g], aux[size_t(g) + 1]));
                    ++nodes;
                }
                for (size_t a = 1; a < k; ++a) RB_CUDA_TRY(order_after(aux[a], stream));
                return cudaSuccess;
            };
            // the big JRPs run their step chains (the solo kernels) one after
            // the other on one branch, beside the table-driven chain of the
            // small ones.  (One branch per big JRP, all concurrent, was slower:
            // the batch workload's 15 JRPs above 10M entries took 1713 ms per
            // step that way and 1500 ms in one chain; the whole batch 2700 ms
            // against 2415 ms.)
            auto big_fork = [&]() -> cudaError_t {
                if (jbig.empty()) return cudaSuccess;
                cudaStream_t st;
                RB_CUDA_TRY(aux_stream(kBigStream0, &st));
                return order_after(stream, st);
            };
            auto big_join = [&]() -> cudaError_t {
                return jbig.empty() ? cudaSuccess : order_after(aux[kBigStream0], stream);
            };
            RB_CUDA_TRY(big_fork());
            for (size_t b = 0; b < jbig.size(); ++b) {
                auto& sv = *j[jbig[b]].s;
                cudaStream_t st = aux[kBigStream0];
                for (int s = 0; s < op_steps; ++s) {
                    auto& dv = sv.d;
                    if (s + 1 < op_steps) {
                        RB_CUDA_TRY((sv.template launch_x<true, false>(dv.xh, dv.yh, dv.zh, s, 0, st)));
                        RB_CUDA_TRY((sv.template launch_yz<true, false>(dv.yh, dv.zh, s, 0, st)));
                    } else {
                        RB_CUDA_TRY((sv.template launch_x<true, true>(dv.xh, dv.yh, dv.zh, s, 0, st)));
                        RB_CUDA_TRY((sv.template launch_yz<true, true>(dv.yh, dv.zh, s, 0, st)));
                    }
                    nodes += 3;
                }
            }
            for (int s = 0; s < op_steps; ++s) {
                const bool last = s + 1 == op_steps;
                RB_CUDA_TRY(x_stage([&](int c, cudaStream_t st) {
                    return last ? launch_x<true, true>(c, s, 0, st) : launch_x<true, false>(c, s, 0, st);
                }));
                RB_CUDA_TRY(yz_stage(
                    [&](cudaStream_t st) { return last ? launch_y<true, true>(s, 0, st) : launch_y<true, false>(s, 0, st); },
                    [&](int c, cudaStream_t st) {
                        return last ? launch_yz<true, true>(c, s, 0, st) : launch_yz<true, false>(c, s, 0, st);
                    }));
            }
            RB_CUDA_TRY(big_join());
            bj_upper<Real><<<sms * 8, pria::kAuxThreads, 0, stream>>>(jdevs.buf.ptr, t_up.buf.ptr, counts.ptr + kUp);
            bj_lower<Real><<<sms * 8, pria::kAuxThreads, 0, stream>>>(jdevs.buf.ptr, t_jlow.buf.ptr, counts.ptr + kJLow);
            bj_check<Real><<<sms * 4, pria::kCheckBlock, 0, stream>>>(jdevs.buf.ptr, jmeta.buf.ptr, l_jcheck.buf.ptr,
                                                                     counts.ptr + kJCheck, 1);
            nodes += 3;
            // the gated restart step: big ones on their branches, small ones by tables
            RB_CUDA_TRY(big_fork());
            for (size_t b = 0; b < jbig.size(); ++b) {
                auto& sv = *j[jbig[b]].s;
                auto& dv = sv.d;
                cudaStream_t st = aux[kBigStream0];
                RB_CUDA_TRY((sv.template launch_x<false, true>(dv.x2s, dv.y2s, dv.z2s, 0, 1, st)));
                RB_CUDA_TRY((sv.template launch_yz<false, true>(dv.y2s, dv.z2s, 0, 1, st)));
                nodes += 3;
            }
            RB_CUDA_TRY(x_stage([&](int c, cudaStream_t st) { return launch_x<false, true>(c, 0, 1, st); }));
            RB_CUDA_TRY(yz_stage([&](cudaStream_t st) { return launch_y<false, true>(0, 1, st); },
                                 [&](int c, cudaStream_t st) { return launch_yz<false, true>(c, 0, 1, st); }));
            RB_CUDA_TRY(big_join());
            bj_check<Real><<<sms * 4, pria::kCheckBlock, 0, stream>>>(jdevs.buf.ptr, jmeta.buf.ptr, l_jcheck.buf.ptr,
                                                                     counts.ptr + kJCheck, 2);
            nodes += 1;
        }
        if (hq && hj) RB_CUDA_TRY(order_after(sq, stream));
        const int slots = int(ids.size());
        b_gather<Real><<<std::max(1, ceil_div(int(q.size() + j.size()), 128)), 128, 0, stream>>>(
            qdevs.buf.ptr, qid_t.buf.ptr, int(q.size()), jdevs.buf.ptr, jid_t.buf.ptr, int(j.size()), live.buf.ptr,
            summary.ptr);
        nodes += 1;
        RB_CUDA_TRY(cudaMemcpyAsync(hsummary, summary.ptr, sizeof(Summary) * slots, cudaMemcpyDeviceToHost, stream));
        block_nodes = nodes;
        return cudaGetLastError();
    }

    int capture() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        if (set_attributes()) return -int(cudaErrorUnknown);
        // every auxiliary stream and fork/join event exists before the capture
        int ex = 0, eg = 0;
        for (bool b : xclasses) ex += b;
        for (bool b : groups) eg += b;
        const size_t wide = std::max(size_t(std::max(ex, eg)) + 1, kBigStream0 + (jbig.empty() ? 0 : 1));
        const size_t events_needed =
            2 + size_t(op_steps + 1) * 2 * size_t(std::max(0, ex - 1) + eg) + 4;
        cudaStream_t tmp;
        if (aux_stream(wide, &tmp)) return -int(cudaErrorUnknown);
        while (fj.size() < events_needed) {
            cudaEvent_t ev;
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) return -int(cudaErrorUnknown);
            fj.push_back(ev);
        }
        if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal)) return -int(cudaErrorUnknown);
        const cudaError_t st = enqueue_block();
        const cudaError_t st2 = cudaStreamEndCapture(stream, &graph);
        if (st || st2) return -int(st ? st : st2);
        if (cudaGraphInstantiate(&exec, graph, 0)) return -int(cudaErrorUnknown);
        dirty = false;
        return 0;
    }

    // Cold-start the instances added since the last call.  Their first step
    // and check run on the layout stream, so the blocks already queued keep
    // the GPU busy meanwhile (no drain): the engine's stream then waits for
    // the layout stream, and the tables (uploaded on the engine's stream,
    // behind the queued blocks) take the newcomers in from the next capture.
    int start() override {
        for (auto& qi : q) {
            if (!qi.s || qi.started) continue;
            qi.s->stream = lay;
            const int st = qi.s->start_solve();
            qi.s->stream = stream;
            if (st) return st;
            if (joined(qi.s->stream)) return PRAQ_ERROR_CUDA;
            qi.started = true;
            qi.join = launched;
            nlaunch += qi.s->launches();
            qi.done = qi.s->mirror->terminated != 0;
            const auto* c = qi.s->mirror;
            qi.last = Summary{c->lower, c->upper, c->gap, c->iteration, c->terminated, 0};
        }
        for (auto& ji : j) {
            if (!ji.s || ji.started) continue;
            ji.s->stream = lay;
            const cudaError_t st = ji.s->start_solve();
            ji.s->stream = stream;
            if (st) return -int(st);
            if (joined(ji.s->stream)) return -int(cudaErrorUnknown);
            ji.started = true;
            ji.join = launched;
            nlaunch += ji.s->launches();
            ji.done = ji.s->mirror->terminated != 0;
            const auto* c = ji.s->mirror;
            ji.last = Summary{c->lower, c->upper, c->gap, c->iteration, c->terminated, 0};
        }
        return rebuild();
    }

    int active() const {
        int a = 0;
        for (auto& qi : q) a += qi.s && qi.started && !qi.done;
        for (auto& ji : j) a += ji.s && ji.started && !ji.done;
        return a;
    }

    // A new capture does not wait for the blocks in flight: they replay the
    // old executable graph (freed when they finish), whose tables and slots
    // stay valid (tables are rewritten on the stream behind them, summaries
    // are written at instance ids).
    int launch() override {
        if (dirty) {
            const int rc = capture();
            if (rc) return rc;
        }
        if (pending >= int(events.size())) return -int(cudaErrorNotReady);
        if (cudaGraphLaunch(exec, stream)) return -int(cudaErrorUnknown);
        if (cudaEventRecord(events[(head + pending) % events.size()], stream)) return -int(cudaErrorUnknown);
        ++pending;
        ++launched;
        nlaunch += block_nodes;
        return 0;
    }

    // Wait for every enqueued block (without retiring anything new).
    int drain() {
        if (cudaStreamSynchronize(stream)) return -1;
        head = (head + pending) % int(events.size());
        synced += pending;
        pending = 0;
        bury(true);
        return 0;
    }

    // Removed instances whose memory blocks still in flight may read (their
    // control blocks and descriptors: those blocks skip them, but look);
    // each is freed once every block enqueued before its removal has been
    // synced.  Freed on the layout stream, so the host never waits for the
    // engine's stream here.
    struct Grave {
        std::unique_ptr<praq::Solver<Real>> qs;
        std::unique_ptr<pria::Solver<Real>> js;
        long long after;   // blocks that must have been synced first
    };
    std::vector<Grave> graves;
    void bury(bool all) {
        for (size_t g = 0; g < graves.size();) {
            if (all || graves[g].after <= synced) {
                if (graves[g].qs) graves[g].qs->stream = lay;
                if (graves[g].js) graves[g].js->stream = lay;
                graves[g].qs.reset();
                graves[g].js.reset();
                graves[g] = std::move(graves.back());
                graves.pop_back();
            } else {
                ++g;
            }
        }
    }

    int sync(int* out_ids, int max, int* count) override {
        if (count) *count = 0;
        if (pending == 0) return active();
        if (cudaEventSynchronize(events[head])) return -int(cudaErrorUnknown);
        head = (head + 1) % int(events.size());
        --pending;
        const long long block = synced++;
        bury(false);
        // the host copy holds the state after this block (or a later one)
        bool changed = false;
        int nout = 0;
        for (int id = 0; id < int(ids.size()); ++id) {
            const auto [kind, k] = ids[id];
            const int slot = id;
            bool* done = kind == 0 ? &q[k].done : &j[k].done;
            const bool running = kind == 0 ? (q[k].s && q[k].started && !q[k].done)
                                           : (j[k].s && j[k].started && !j[k].done);
            if (!running) continue;
            // only blocks enqueued after the instance joined carry its state
            if (block < (kind == 0 ? q[k].join : j[k].join)) continue;
            const Summary s = hsummary[slot];
            (kind == 0 ? q[k].last : j[k].last) = s;
            if (s.terminated) {
                *done = true;
                changed = true;
                if (out_ids && nout < max) out_ids[nout] = id;
                ++nout;
            }
        }
        if (count) *count = std::min(nout, max);
        if (changed) {
            // blocks already enqueued see the flag and skip the retired
            // instances; the next ones run without their tiles
            const int rc = rebuild();
            if (rc) return rc;
        }
        return active();
    }

    int inflight() const override { return pending; }

    int run(int64_t max_blocks) override {
        int64_t blocks = 0;
        while (active() > 0 && (max_blocks < 0 || blocks < max_blocks)) {
            while (pending < 2 && (max_blocks < 0 || blocks + pending < max_blocks)) {
                const int rc = launch();
                if (rc) return rc;
            }
            const int rc = sync(nullptr, 0, nullptr);
            if (rc < 0) return rc;
            ++blocks;
        }
        return drain();
    }

    int status(int id, int* done, int64_t* it, double* lo, double* up) override {
        if (id < 0 || id >= int(ids.size())) return PRAQ_ERROR_ARGUMENT;
        const auto [kind, k] = ids[id];
        const Summary& s = kind == 0 ? q[k].last : j[k].last;
        if (done) *done = kind == 0 ? q[k].done : j[k].done;
        if (it) *it = s.iteration;
        if (lo) *lo = s.lower;
        if (up) *up = s.upper;
        return 0;
    }

    // A finished instance is read on the layout stream, with no wait for the
    // blocks in flight: they skip it and write none of its memory, and the
    // block that finished it is complete (the summary that said so was copied
    // at its end).  An instance still running is read after a drain.
    int result_qubo(int id, double* x, PraqResult* r) override {
        if (id < 0 || id >= int(ids.size()) || ids[id].first != 0) return PRAQ_ERROR_ARGUMENT;
        auto& qi = q[ids[id].second];
        if (!qi.s) return PRAQ_ERROR_ARGUMENT;
        if (!qi.done && pending && drain()) return PRAQ_ERROR_CUDA;
        const cudaStream_t on = qi.done ? lay : stream;
        if (cudaMemcpyAsync(qi.s->mirror, qi.s->d.ctl, sizeof(praq::Control), cudaMemcpyDeviceToHost, on) ||
            cudaStreamSynchronize(on))
            return PRAQ_ERROR_CUDA;
        qi.s->stream = on;
        const int st = qi.s->result(x, nullptr, r);
        qi.s->stream = stream;
        return st;
    }

    int set_warm_qubo(int id, const double* x, const double* y2) override {
        if (id < 0 || id >= int(ids.size()) || ids[id].first != 0) return PRAQ_ERROR_ARGUMENT;
        auto& qi = q[ids[id].second];
        if (!qi.s || qi.started) return PRAQ_ERROR_ARGUMENT;
        // on the layout stream, where the instance will be started
        qi.s->stream = lay;
        const int st = qi.s->set_warm(x, y2);
        qi.s->stream = stream;
        return st;
    }

    // The point of the instance's last check (its bracket's primal and dual),
    // in instance units, whether or not it has terminated.
    int point_qubo(int id, double* x, double* y2) override {
        if (id < 0 || id >= int(ids.size()) || ids[id].first != 0) return PRAQ_ERROR_ARGUMENT;
        auto& qi = q[ids[id].second];
        if (!qi.s || !qi.started) return PRAQ_ERROR_ARGUMENT;
        if (pending && drain()) return PRAQ_ERROR_CUDA;
        if (cudaMemcpyAsync(qi.s->mirror, qi.s->d.ctl, sizeof(praq::Control), cudaMemcpyDeviceToHost, stream) ||
            cudaStreamSynchronize(stream))
            return PRAQ_ERROR_CUDA;
        return qi.s->result(x, y2, nullptr);
    }

    int result_jrp(int id, double* x, double* y, double* z, pria_result_info* info) override {
        if (id < 0 || id >= int(ids.size()) || ids[id].first != 1) return int(cudaErrorInvalidValue);
        auto& ji = j[ids[id].second];
        if (!ji.s) return int(cudaErrorInvalidValue);
        if (!ji.done && pending && drain()) return int(cudaErrorUnknown);
        const cudaStream_t on = ji.done ? lay : stream;
        if (cudaMemcpyAsync(ji.s->mirror, ji.s->d.ctl, sizeof(pria::Control), cudaMemcpyDeviceToHost, on) ||
            cudaStreamSynchronize(on))
            return int(cudaErrorUnknown);
        ji.s->stream = on;
        const int st = ji.s->result(x, y, z, info);
        ji.s->stream = stream;
        return st;
    }

    // A running instance leaves the work tables first (after the blocks in
    // flight have finished); then its device memory is freed.  A finished
    // one (or one never started) is out of the tables already: its memory is
    // freed once the blocks now in flight have been synced, with no wait.
    int remove(int id) override {
        if (id < 0 || id >= int(ids.size())) return PRAQ_ERROR_ARGUMENT;
        const auto [kind, k] = ids[id];
        const bool running = kind == 0 ? (q[k].s && q[k].started && !q[k].done)
                                       : (j[k].s && j[k].started && !j[k].done);
        if (running) {
            if (pending && drain()) return PRAQ_ERROR_CUDA;
            if (kind == 0) q[k].s.reset(); else j[k].s.reset();
            return rebuild();
        }
        if (pending) {
            Grave g{};
            if (kind == 0) g.qs = std::move(q[k].s); else g.js = std::move(j[k].s);
            g.after = launched;
            graves.push_back(std::move(g));
        } else if (kind == 0) {
            q[k].s.reset();
        } else {
            j[k].s.reset();
        }
        return 0;
    }

    int64_t device_bytes() const override {
        int64_t b = 0;
        for (auto& qi : q) if (qi.s) b += int64_t(qi.s->device_bytes());
        for (auto& ji : j) if (ji.s) b += int64_t(ji.s->device_bytes());
        return b;
    }

    int apply_shapes(const Shapes& sh) {
        shapes = sh;
        dirty = true;
        return 0;
    }

    int set_shapes(const reform_shapes& s) override {
        Shapes sh = shapes;
        if (s.grid_multiplier > 0) sh.grid_mult = std::min(16, std::max(1, s.grid_multiplier));
        shapes_fixed = true;
        if (pending && drain()) return PRAQ_ERROR_CUDA;
        const int rc = apply_shapes(sh);
        return rc ? rc : rebuild();
    }

    int restart() override { return restart_all(); }

    // Restart every instance from its cold start (the tuner, repeated solves).
    int restart_all() {
        if (pending && drain()) return -1;
        for (auto& qi : q) if (qi.s) qi.started = qi.done = false;
        for (auto& ji : j) if (ji.s) ji.started = ji.done = false;
        return start();
    }

    std::tuple<int, int, int, int, int> size_class() const {
        long long m = 0, nd = 0;
        int nq = 0, nj = 0;
        for (auto& qi : q) if (qi.s) { m += qi.s->m; ++nq; }
        for (auto& ji : j) if (ji.s) { nd += ji.s->d.nd; ++nj; }
        auto lg = [](long long v) { int b = 0; while (v > 1) { v >>= 1; ++b; } return b; };
        return {nq > 0 ? lg(nq) + 1 : 0, lg(m), nj > 0 ? lg(nj) + 1 : 0, lg(nd), int(sizeof(Real))};
    }

    // Time one block per candidate shape on this batch's own instances and keep
    // the fastest; remembered per size class for later batches.
    int autotune(reform_shapes* out) override {
        const auto key = size_class();
        {
            std::lock_guard<std::mutex> lock(tuned_mu);
            auto it = tuned.find(key);
            if (it != tuned.end()) {
                const int rc = apply_shapes(it->second);
                if (!rc && out) out->grid_multiplier = it->second.grid_mult;
                return rc ? rc : restart_all();
            }
        }
        std::vector<Shapes> cands;
        for (int gm : {2, 4, 8, 16}) cands.push_back(Shapes{gm});
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) || cudaEventCreate(&b)) return -1;
        float best = 1e30f;
        Shapes pick = shapes;
        for (auto& c : cands) {
            if (apply_shapes(c) || restart_all()) return -1;
            if (dirty && capture()) return -1;
            // one untimed block (first touch), then one timed
            if (cudaGraphLaunch(exec, stream) || cudaStreamSynchronize(stream)) return -1;
            if (cudaEventRecord(a, stream) || cudaGraphLaunch(exec, stream) || cudaEventRecord(b, stream) ||
                cudaEventSynchronize(b))
                return -1;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            nlaunch += 2 * block_nodes;
            if (ms < best) {
                best = ms;
                pick = c;
            }
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        {
            std::lock_guard<std::mutex> lock(tuned_mu);
            tuned[key] = pick;
        }
        if (out) out->grid_multiplier = pick.grid_mult;
        if (apply_shapes(pick)) return -1;
        return restart_all();
    }

    int64_t launches() const override { return nlaunch; }
};

}  // namespace
}  // namespace batch
}  // namespace rb200

using namespace rb200;

struct reform_batch {
    std::unique_ptr<batch::EngineBase> impl;
};

extern "C" {

int reform_batch_create(int use_float32, void* stream, reform_batch** out) {
    if (!out) return PRAQ_ERROR_ARGUMENT;
    *out = nullptr;
    auto b = std::make_unique<reform_batch>();
    int rc;
    if (use_float32) {
        auto* e = new batch::Engine<float>();
        b->impl.reset(e);
        rc = e->init(static_cast<cudaStream_t>(stream));
    } else {
        auto* e = new batch::Engine<double>();
        b->impl.reset(e);
        rc = e->init(static_cast<cudaStream_t>(stream));
    }
    if (rc) return rc;
    *out = b.release();
    return 0;
}

int reform_batch_add_qubo(reform_batch* b, const PraqInstance* instance, const PraqParameters* parameters) {
    if (!b || !instance || !parameters) return PRAQ_ERROR_ARGUMENT;
    const int64_t limit = std::numeric_limits<int>::max();
    if (instance->n <= 0 || instance->n > limit / 32 || instance->m < 0 || instance->m > limit / 2)
        return PRAQ_ERROR_INSTANCE;
    if (!instance->diag || (instance->m > 0 && (!instance->rows || !instance->cols || !instance->vals)))
        return PRAQ_ERROR_INSTANCE;
    return b->impl->add_qubo(*instance, *parameters);
}

int reform_batch_add_jrp(reform_batch* b, int64_t n, int64_t t, const double* k, double k0, const double* h,
                         const pria_params* params) {
    if (!b || !params) return -int(cudaErrorInvalidValue);
    return b->impl->add_jrp(n, t, k, k0, h, *params);
}

int reform_batch_add_jrp_demand(reform_batch* b, int64_t n, int64_t t, const double* k, double k0,
                                const double* rate, const double* demand, const pria_params* params) {
    if (!b || !params) return -int(cudaErrorInvalidValue);
    return b->impl->add_jrp_demand(n, t, k, k0, rate, demand, *params);
}

int reform_batch_start(reform_batch* b) { return b ? b->impl->start() : PRAQ_ERROR_ARGUMENT; }
int reform_batch_run(reform_batch* b, int64_t max_blocks) { return b ? b->impl->run(max_blocks) : PRAQ_ERROR_ARGUMENT; }
int reform_batch_launch(reform_batch* b) { return b ? b->impl->launch() : PRAQ_ERROR_ARGUMENT; }
int reform_batch_sync(reform_batch* b, int* ids, int max, int* count) {
    return b ? b->impl->sync(ids, max, count) : PRAQ_ERROR_ARGUMENT;
}
int reform_batch_inflight(const reform_batch* b) { return b ? b->impl->inflight() : 0; }
int reform_batch_status(reform_batch* b, int id, int* done, int64_t* iterations, double* lower, double* upper) {
    return b ? b->impl->status(id, done, iterations, lower, upper) : PRAQ_ERROR_ARGUMENT;
}
int reform_batch_result_qubo(reform_batch* b, int id, double* x, PraqResult* result) {
    return b ? b->impl->result_qubo(id, x, result) : PRAQ_ERROR_ARGUMENT;
}
int reform_batch_result_jrp(reform_batch* b, int id, double* x, double* y, double* z, pria_result_info* info) {
    return b ? b->impl->result_jrp(id, x, y, z, info) : PRAQ_ERROR_ARGUMENT;
}
int reform_batch_remove(reform_batch* b, int id) { return b ? b->impl->remove(id) : PRAQ_ERROR_ARGUMENT; }
int reform_batch_set_warm_qubo(reform_batch* b, int id, const double* x, const double* y2) {
    return b ? b->impl->set_warm_qubo(id, x, y2) : PRAQ_ERROR_ARGUMENT;
}
int reform_batch_point_qubo(reform_batch* b, int id, double* x, double* y2) {
    return b ? b->impl->point_qubo(id, x, y2) : PRAQ_ERROR_ARGUMENT;
}
int64_t reform_batch_device_bytes(const reform_batch* b) { return b ? b->impl->device_bytes() : 0; }
int reform_batch_set_shapes(reform_batch* b, const reform_shapes* s) {
    return b && s ? b->impl->set_shapes(*s) : PRAQ_ERROR_ARGUMENT;
}
int reform_batch_autotune(reform_batch* b, reform_shapes* out) { return b ? b->impl->autotune(out) : PRAQ_ERROR_ARGUMENT; }
int reform_batch_restart(reform_batch* b) { return b ? b->impl->restart() : PRAQ_ERROR_ARGUMENT; }
int64_t reform_batch_launches(const reform_batch* b) { return b ? b->impl->launches() : 0; }
void reform_batch_destroy(reform_batch* b) { delete b; }

}  // extern "C"
