// server.cu -- the continuous-batching request loop behind the C ABI
// (include/reform.h, reform_server_*).
//
// A server owns a batched engine (reform_batch_*; two of them with FP32
// iterates: the FP32 engine and the FP64 engine that stalled QUBOs continue
// in) and one host thread that drives them:
//
//   * submit copies a request's instance into host memory the server owns and
//     queues it; the caller's arrays are free as soon as submit returns;
//   * the loop admits queued requests in arrival order while the device
//     budget allows (each request reserves an estimate of the bytes its layout
//     and iterates take; the first request is always admitted), lays them out
//     and cold-starts them between two block replays, and keeps
//     `blocks_in_flight` op_steps blocks queued on the GPU;
//   * after each block it reads every instance's control block (one copy),
//     marks the converged requests finished (their iterates stay on the
//     device) and wakes pollers; a QUBO whose FP32 gap has not halved over
//     `stall_iterations` iterations moves to the FP64 engine, warm-started at
//     its last check;
//   * the caller polls for finished ids, reads results (bounds, iterations,
//     the primal; a JRP's x, y, z) and retires them, which returns their
//     device memory and their share of the budget.
//
// No counterpart in the reference, whose solvers take one instance per call
// (praq_solve) or fan independent solves out to host threads
// (pria_solve_batch_*, jrp/pria-cuda/src/pria.cu:15-44); the pattern of a
// library-owned worker behind a C call is the same as the latter's.
//
// Threading: `mu` guards the request table and the queues, `emu` the
// engines (which are not thread-safe).  Lock order: emu before mu.  The loop
// takes `emu` around its engine calls, so a caller's result read waits at
// most about one block.
#include "../../include/reform.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace rb200 {
namespace server {
namespace {

using Clock = std::chrono::steady_clock;

enum Kind { kQubo = 0, kJrp = 1, kJrpDemand = 2 };
enum State { kWaiting = 0, kRunning = 1, kFinished = 2, kFailed = 3 };

struct Request {
    int64_t id = 0;
    int kind = kQubo;
    // the instance, owned
    int64_t n = 0, m = 0, t = 0;
    double k0 = 0.0;
    std::vector<double> diag, vals, k, h, rate, demand;
    std::vector<int64_t> rows, cols;
    int64_t need = 0;                    // reserved device bytes
    double arrival = 0.0, admitted = -1.0, finished = -1.0;
    int state = kWaiting;
    int error = 0;                       // the engine's error for a failed request
    int engine = 0, eid = -1;
    // FP32 plateau tracking (QUBOs in the FP32 engine)
    double ref_gap = INFINITY;
    int64_t ref_it = 0;
    int64_t carried = 0;                 // FP32 iterations before an escalation
    bool stalled = false;                // to move to the FP64 engine
    double lower = NAN, upper = NAN;
    int64_t iterations = 0;
};

// Device bytes a request holds once laid out: its iterates, layout and partial
// sums, a little above the solvers' own counts.
int64_t footprint(const Request& r, int use_float32) {
    const int64_t R = use_float32 ? 4 : 8;
    if (r.kind == kQubo)
        return r.m * (12 + 7 * R) + r.n * (8 + 6 * R) + (r.n * 32 + r.m) / 64 * 64 + 4096;
    const int64_t tp = r.t + (r.t & 1);
    const int64_t nd = r.n * tp * (tp + 1) / 2;
    return nd * 13 * R + r.n * tp * 16 + 65536;
}

}  // namespace

struct Server {
    reform_server_options opt{};
    PraqParameters qp{}, qp64{};
    pria_params jp{};
    reform_batch* eng[2] = {nullptr, nullptr};
    std::mutex mu, emu;
    std::condition_variable cv_work, cv_done;
    std::deque<int64_t> incoming, waiting;
    std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
    std::unordered_map<int, int64_t> by_eid[2];
    std::deque<int64_t> finished;        // not yet polled
    std::vector<int64_t> retiring;       // retired by the caller, removal pending
    int64_t next_id = 0, reserved = 0, high_water = 0;
    int running = 0;
    int64_t completed = 0;
    bool stop = false;
    int sticky = 0;                      // an engine error: the loop has stopped
    Clock::time_point t0 = Clock::now();
    std::thread loop;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

    int engine_for(int which) {
        if (eng[which]) return 0;
        const int use_float32 = which == 0 ? opt.use_float32 : 0;
        return reform_batch_create(use_float32, nullptr, &eng[which]);
    }

    // Stops the loop on an engine error (called with emu held).
    void fail(int st) {
        std::lock_guard<std::mutex> lock(mu);
        sticky = st ? st : -1;
        stop = true;
        cv_done.notify_all();
    }

    // --- loop-side work (engine calls under emu) -------------------------

    // Lay out and start the requests taken for admission.
    void admit(const std::vector<Request*>& batch) {
        std::lock_guard<std::mutex> elock(emu);
        bool any = false;
        for (Request* r : batch) {
            int eid;
            if (r->kind == kQubo) {
                const PraqInstance view{r->n, r->m, r->diag.data(), r->rows.data(), r->cols.data(),
                                        r->vals.data()};
                eid = reform_batch_add_qubo(eng[0], &view, &qp);
            } else if (r->kind == kJrp) {
                eid = reform_batch_add_jrp(eng[0], r->n, r->t, r->k.data(), r->k0, r->h.data(), &jp);
            } else {
                eid = reform_batch_add_jrp_demand(eng[0], r->n, r->t, r->k.data(), r->k0, r->rate.data(),
                                                  r->demand.data(), &jp);
            }
            std::lock_guard<std::mutex> lock(mu);
            r->admitted = now();
            if (eid < 0) {
                r->state = kFailed;
                r->error = eid;
                r->finished = r->admitted;
                reserved -= r->need;
                finished.push_back(r->id);
                cv_done.notify_all();
                continue;
            }
            r->engine = 0;
            r->eid = eid;
            r->state = kRunning;
            by_eid[0][eid] = r->id;
            ++running;
            any = true;
        }
        if (any) {
            const int st = reform_batch_start(eng[0]);
            if (st) fail(st);
        }
        // requests that finished at their cold start never enter a block
        collect(0);
    }

    // Requests of engine `which` that have terminated become finished (their
    // iterates stay on the device until retired); FP32 QUBOs on a plateau
    // are marked for the FP64 engine.
    void collect(int which) {
        if (!eng[which]) return;
        std::vector<std::pair<int, int64_t>> live;
        {
            std::lock_guard<std::mutex> lock(mu);
            for (auto& kv : by_eid[which])
                if (reqs.at(kv.second)->state == kRunning) live.emplace_back(kv.first, kv.second);
        }
        bool woke = false;
        for (auto& [eid, rid] : live) {
            int done = 0;
            int64_t it = 0;
            double lo = NAN, up = NAN;
            if (reform_batch_status(eng[which], eid, &done, &it, &lo, &up)) continue;
            std::lock_guard<std::mutex> lock(mu);
            Request& r = *reqs.at(rid);
            if (done) {
                r.state = kFinished;
                r.finished = now();
                r.lower = lo;
                r.upper = up;
                r.iterations = it + r.carried;
                --running;
                ++completed;
                finished.push_back(rid);
                woke = true;
            } else if (which == 0 && opt.use_float32 && r.kind == kQubo && opt.stall_iterations > 0) {
                const double gap = (up - lo) / (1.0 + std::fabs(up) + std::fabs(lo));
                if (!(gap > 0.5 * r.ref_gap)) {          // halved (or the first look)
                    r.ref_gap = gap;
                    r.ref_it = it;
                } else if (it - r.ref_it >= opt.stall_iterations) {
                    r.stalled = true;
                }
            }
        }
        if (woke) cv_done.notify_all();
    }

    // A stalled FP32 QUBO continues in the FP64 engine from its last check.
    void escalate(Request& r) {
        int done = 0;
        int64_t it = 0;
        double lo, up;
        reform_batch_status(eng[0], r.eid, &done, &it, &lo, &up);
        std::vector<double> x(size_t(r.n)), y(size_t(2 * std::max<int64_t>(r.m, 1)));
        int st = reform_batch_point_qubo(eng[0], r.eid, x.data(), y.data());
        if (!st) st = reform_batch_remove(eng[0], r.eid);
        if (!st) st = engine_for(1);
        int e64 = -1;
        if (!st) {
            const PraqInstance view{r.n, r.m, r.diag.data(), r.rows.data(), r.cols.data(), r.vals.data()};
            e64 = reform_batch_add_qubo(eng[1], &view, &qp64);
            if (e64 < 0) st = e64;
        }
        if (!st) st = reform_batch_set_warm_qubo(eng[1], e64, x.data(), y.data());
        if (!st) st = reform_batch_start(eng[1]);
        std::lock_guard<std::mutex> lock(mu);
        by_eid[0].erase(r.eid);
        r.stalled = false;
        if (st) {
            r.state = kFailed;
            r.error = st;
            r.finished = now();
            r.eid = -1;
            reserved -= r.need;   // its device memory went with the removal
            --running;
            finished.push_back(r.id);
            cv_done.notify_all();
            return;
        }
        r.carried = it;
        r.engine = 1;
        r.eid = e64;
        by_eid[1][e64] = r.id;
    }

    // Requests the caller retired: their device memory and budget share back.
    void remove_retired(const std::vector<int64_t>& ids) {
        std::lock_guard<std::mutex> elock(emu);
        for (int64_t rid : ids) {
            std::unique_ptr<Request> r;
            {
                std::lock_guard<std::mutex> lock(mu);
                auto it = reqs.find(rid);
                if (it == reqs.end()) continue;
                r = std::move(it->second);
                reqs.erase(it);
                if (r->eid >= 0) by_eid[r->engine].erase(r->eid);
                if (r->state == kRunning) --running;                // cancelled while running
                if (r->state != kFailed) reserved -= r->need;       // a failed one gave it back already
            }
            if (r->eid >= 0 && (r->state == kRunning || r->state == kFinished))
                reform_batch_remove(eng[r->engine], r->eid);
        }
    }

    bool engine_has_work(int which) {
        std::lock_guard<std::mutex> lock(mu);
        for (auto& kv : by_eid[which])
            if (reqs.at(kv.second)->state == kRunning) return true;
        return false;
    }

    void run() {
        int since_admit = 1 << 30;
        for (;;) {
            std::vector<Request*> admits;
            std::vector<int64_t> retire_now;
            {
                std::unique_lock<std::mutex> lock(mu);
                cv_work.wait(lock, [&] {
                    return stop || running > 0 || !incoming.empty() || !retiring.empty() || !waiting.empty();
                });
                if (stop) break;
                while (!incoming.empty()) {
                    waiting.push_back(incoming.front());
                    incoming.pop_front();
                }
                // while requests run, admission and removal happen at most
                // every `admit_every` blocks
                const bool turn = running == 0 || since_admit >= opt.admit_every;
                if (turn && !retiring.empty()) retire_now.swap(retiring);
                while (turn && !waiting.empty()) {
                    Request* r = reqs.at(waiting.front()).get();
                    const int64_t after = reserved + r->need;
                    const bool first = running == 0 && admits.empty();
                    if (!first && after > opt.budget_bytes) break;
                    reserved = after;
                    high_water = std::max(high_water, reserved);
                    admits.push_back(r);
                    waiting.pop_front();
                }
            }
            if (!retire_now.empty()) remove_retired(retire_now);
            if (!admits.empty()) {
                since_admit = 0;
                admit(admits);
            }
            {
                std::lock_guard<std::mutex> lock(mu);
                if (stop) break;
                if (running == 0) continue;
            }
            {
                std::lock_guard<std::mutex> elock(emu);
                int st = 0;
                for (int which = 0; which < 2 && !st; ++which) {
                    if (!eng[which] || !engine_has_work(which)) continue;
                    while (!st && reform_batch_inflight(eng[which]) < opt.blocks_in_flight)
                        st = reform_batch_launch(eng[which]);
                }
                for (int which = 0; which < 2 && !st; ++which) {
                    if (!eng[which] || !reform_batch_inflight(eng[which])) continue;
                    int count = 0;
                    const int active = reform_batch_sync(eng[which], nullptr, 0, &count);
                    if (active < 0) st = active;
                    else collect(which);
                }
                if (st) {
                    fail(st);
                } else {
                    std::vector<Request*> moves;
                    {
                        std::lock_guard<std::mutex> lock(mu);
                        for (auto& kv : by_eid[0]) {
                            Request* r = reqs.at(kv.second).get();
                            if (r->state == kRunning && r->stalled) moves.push_back(r);
                        }
                    }
                    for (Request* r : moves) escalate(*r);
                }
            }
            ++since_admit;
        }
        std::lock_guard<std::mutex> elock(emu);
        for (auto* e : eng)
            if (e)
                while (reform_batch_inflight(e) > 0 && reform_batch_sync(e, nullptr, 0, nullptr) >= 0) {
                }
    }
};

}  // namespace server
}  // namespace rb200

using rb200::server::Request;
using rb200::server::Server;

struct reform_server {
    std::unique_ptr<Server> impl;
};

namespace {

int64_t enqueue(reform_server* s, std::unique_ptr<Request> r) {
    Server& S = *s->impl;
    std::lock_guard<std::mutex> lock(S.mu);
    if (S.stop) return S.sticky ? -std::abs(S.sticky) : PRAQ_ERROR_ARGUMENT;
    r->id = S.next_id++;
    r->arrival = S.now();
    r->need = rb200::server::footprint(*r, S.opt.use_float32);
    const int64_t id = r->id;
    S.reqs[id] = std::move(r);
    S.incoming.push_back(id);
    S.cv_work.notify_one();
    return id;
}

// The finished request `id` of the given kind (0 QUBO, 1 JRP), or null.
Request* finished_request(Server& S, int64_t id, int kind) {
    auto it = S.reqs.find(id);
    if (it == S.reqs.end()) return nullptr;
    Request* r = it->second.get();
    if ((kind == 0) != (r->kind == rb200::server::kQubo)) return nullptr;
    return r->state == rb200::server::kFinished ? r : nullptr;
}

}  // namespace

extern "C" {

reform_server_options reform_server_default_options(void) {
    reform_server_options o{};
    o.budget_bytes = int64_t(150) * 1000 * 1000 * 1000;
    o.tolerance = 1e-4;
    o.max_iter = 200000;
    o.use_float32 = 1;
    o.blocks_in_flight = 2;
    o.admit_every = 4;
    o.stall_iterations = 384;
    return o;
}

int reform_server_create(const reform_server_options* options, reform_server** out) {
    if (!out) return PRAQ_ERROR_ARGUMENT;
    *out = nullptr;
    reform_server_options o = options ? *options : reform_server_default_options();
    const reform_server_options d = reform_server_default_options();
    if (o.budget_bytes <= 0) o.budget_bytes = d.budget_bytes;
    if (!(o.tolerance > 0.0)) o.tolerance = d.tolerance;
    if (o.max_iter == 0) o.max_iter = d.max_iter;
    if (o.blocks_in_flight < 1) o.blocks_in_flight = d.blocks_in_flight;
    if (o.blocks_in_flight > 4) o.blocks_in_flight = 4;   // the engine's ring of enqueued blocks
    if (o.admit_every < 1) o.admit_every = d.admit_every;
    auto s = std::make_unique<reform_server>();
    s->impl = std::make_unique<Server>();
    Server& S = *s->impl;
    S.opt = o;
    S.qp = praq_default_parameters();
    S.qp.tolerance = o.tolerance;
    S.qp.max_iter = o.max_iter;
    S.qp.use_float32 = o.use_float32 ? 1 : 0;
    S.qp64 = S.qp;
    S.qp64.use_float32 = 0;
    S.jp = pria_params_auto(o.max_iter, o.tolerance);
    const int st = S.engine_for(0);
    if (st) return st;
    S.loop = std::thread([&S] { S.run(); });
    *out = s.release();
    return 0;
}

int64_t reform_server_submit_qubo(reform_server* s, const PraqInstance* in) {
    if (!s || !in || in->n <= 0 || in->m < 0 || !in->diag ||
        (in->m > 0 && (!in->rows || !in->cols || !in->vals)))
        return PRAQ_ERROR_ARGUMENT;
    auto r = std::make_unique<Request>();
    r->kind = rb200::server::kQubo;
    r->n = in->n;
    r->m = in->m;
    r->diag.assign(in->diag, in->diag + in->n);
    r->rows.assign(in->rows, in->rows + in->m);
    r->cols.assign(in->cols, in->cols + in->m);
    r->vals.assign(in->vals, in->vals + in->m);
    return enqueue(s, std::move(r));
}

int64_t reform_server_submit_jrp(reform_server* s, int64_t n, int64_t t, const double* order_costs,
                                 double joint_cost, const double* holding_costs) {
    if (!s || n < 1 || t < 1 || !order_costs || !holding_costs) return PRAQ_ERROR_ARGUMENT;
    auto r = std::make_unique<Request>();
    r->kind = rb200::server::kJrp;
    r->n = n;
    r->t = t;
    r->k0 = joint_cost;
    r->k.assign(order_costs, order_costs + n);
    r->h.assign(holding_costs, holding_costs + size_t(n) * t * t);
    return enqueue(s, std::move(r));
}

int64_t reform_server_submit_jrp_demand(reform_server* s, int64_t n, int64_t t, const double* order_costs,
                                        double joint_cost, const double* rate, const double* demand) {
    if (!s || n < 1 || t < 1 || !order_costs || !rate || !demand) return PRAQ_ERROR_ARGUMENT;
    auto r = std::make_unique<Request>();
    r->kind = rb200::server::kJrpDemand;
    r->n = n;
    r->t = t;
    r->k0 = joint_cost;
    r->k.assign(order_costs, order_costs + n);
    r->rate.assign(rate, rate + n);
    r->demand.assign(demand, demand + size_t(n) * t);
    return enqueue(s, std::move(r));
}

int reform_server_poll(reform_server* s, int64_t* ids, int max, int* count, double wait_seconds) {
    if (!s || !count || (max > 0 && !ids)) return PRAQ_ERROR_ARGUMENT;
    Server& S = *s->impl;
    std::unique_lock<std::mutex> lock(S.mu);
    if (wait_seconds > 0.0 && S.finished.empty() && !S.stop)
        S.cv_done.wait_for(lock, std::chrono::duration<double>(wait_seconds),
                           [&] { return !S.finished.empty() || S.stop; });
    int k = 0;
    while (k < max && !S.finished.empty()) {
        ids[k++] = S.finished.front();
        S.finished.pop_front();
    }
    *count = k;
    return S.sticky ? -std::abs(S.sticky) : 0;
}

int reform_server_status(reform_server* s, int64_t id, reform_server_request* out) {
    if (!s || !out) return PRAQ_ERROR_ARGUMENT;
    Server& S = *s->impl;
    std::lock_guard<std::mutex> lock(S.mu);
    auto it = S.reqs.find(id);
    if (it == S.reqs.end()) return PRAQ_ERROR_ARGUMENT;
    const Request& r = *it->second;
    out->state = r.state;
    out->error = r.error;
    out->kind = r.kind == rb200::server::kQubo ? 0 : 1;
    out->escalated = r.engine == 1 ? 1 : 0;
    out->iterations = r.iterations;
    out->lower = r.lower;
    out->upper = r.upper;
    out->arrival = r.arrival;
    out->admitted = r.admitted;
    out->finished = r.finished;
    out->device_bytes = r.need;
    return 0;
}

int reform_server_result_qubo(reform_server* s, int64_t id, double* x, PraqResult* result) {
    if (!s) return PRAQ_ERROR_ARGUMENT;
    Server& S = *s->impl;
    std::lock_guard<std::mutex> elock(S.emu);   // lock order: emu, then mu
    int engine, eid;
    int64_t carried;
    {
        std::lock_guard<std::mutex> lock(S.mu);
        Request* r = finished_request(S, id, 0);
        if (!r) return PRAQ_ERROR_ARGUMENT;
        engine = r->engine;
        eid = r->eid;
        carried = r->carried;
    }
    PraqResult pr{};
    const int st = reform_batch_result_qubo(S.eng[engine], eid, x, &pr);
    pr.iterations += carried;
    if (result) *result = pr;
    return st;
}

int reform_server_result_jrp(reform_server* s, int64_t id, double* x, double* y, double* z,
                             pria_result_info* info) {
    if (!s) return int(cudaErrorInvalidValue);
    Server& S = *s->impl;
    std::lock_guard<std::mutex> elock(S.emu);
    int engine, eid;
    {
        std::lock_guard<std::mutex> lock(S.mu);
        Request* r = finished_request(S, id, 1);
        if (!r) return int(cudaErrorInvalidValue);
        engine = r->engine;
        eid = r->eid;
    }
    return reform_batch_result_jrp(S.eng[engine], eid, x, y, z, info);
}

int reform_server_retire(reform_server* s, int64_t id) {
    if (!s) return PRAQ_ERROR_ARGUMENT;
    Server& S = *s->impl;
    std::lock_guard<std::mutex> lock(S.mu);
    auto it = S.reqs.find(id);
    if (it == S.reqs.end()) return PRAQ_ERROR_ARGUMENT;
    // still queued (not yet taken for admission): it holds no device memory
    auto w = std::find(S.waiting.begin(), S.waiting.end(), id);
    auto q = std::find(S.incoming.begin(), S.incoming.end(), id);
    if (w != S.waiting.end() || q != S.incoming.end()) {
        if (w != S.waiting.end()) S.waiting.erase(w);
        if (q != S.incoming.end()) S.incoming.erase(q);
        S.reqs.erase(it);
        return 0;
    }
    S.retiring.push_back(id);
    S.cv_work.notify_one();
    return 0;
}

int reform_server_stats(reform_server* s, reform_server_counts* out) {
    if (!s || !out) return PRAQ_ERROR_ARGUMENT;
    Server& S = *s->impl;
    std::lock_guard<std::mutex> elock(S.emu);   // the engines' byte counts
    std::lock_guard<std::mutex> lock(S.mu);
    out->waiting = int64_t(S.waiting.size() + S.incoming.size());
    out->running = S.running;
    out->completed = S.completed;
    out->reserved_bytes = S.reserved;
    out->high_water_bytes = S.high_water;
    out->device_bytes = 0;
    for (auto* e : S.eng)
        if (e) out->device_bytes += reform_batch_device_bytes(e);
    out->error = S.sticky;
    return 0;
}

void reform_server_destroy(reform_server* s) {
    if (!s) return;
    Server& S = *s->impl;
    {
        std::lock_guard<std::mutex> lock(S.mu);
        S.stop = true;
    }
    S.cv_work.notify_all();
    if (S.loop.joinable()) S.loop.join();
    {
        std::lock_guard<std::mutex> elock(S.emu);
        S.reqs.clear();
        for (auto*& e : S.eng) {
            if (e) reform_batch_destroy(e);
            e = nullptr;
        }
    }
    delete s;
}

}  // extern "C"
