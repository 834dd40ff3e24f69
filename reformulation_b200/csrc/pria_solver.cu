// pria_solver.cu -- the C ABI of the PRIA solver (include/pria.h); the
// solver itself (kernels, device layout, host driver) is pria_core.cuh.
#include "pria_core.cuh"
#include "../../include/reform.h"

using namespace rb200;

struct reform_pria_solver {
    std::unique_ptr<pria::SolverBase> impl;
};

namespace {

template <class T>
static int solve_one(int64_t n, int64_t t, const T* k, T k0, const T* h, const pria_params* params,
                     const T* wx, const T* wy, const T* wz, T* x, T* y, T* z, pria_result_info* info,
                     int use_float32) {
    std::unique_ptr<pria::SolverBase> impl;
    int st = pria::create<T>(n, t, k, double(k0), h, params, use_float32, nullptr, impl);
    if (st) return st;
    if (wx && wy && wz) {
        const size_t full = size_t(n) * size_t(t) * size_t(t);
        std::vector<double> a(wx, wx + full), b(wy, wy + full), c(wz, wz + full);
        if ((st = impl->set_warm(a.data(), b.data(), c.data()))) return st;
    }
    if ((st = impl->run())) return st;
    if constexpr (sizeof(T) == 8) {
        return impl->result(reinterpret_cast<double*>(x), reinterpret_cast<double*>(y),
                            reinterpret_cast<double*>(z), info);
    } else {
        return impl->result_f32(reinterpret_cast<float*>(x), reinterpret_cast<float*>(y),
                                reinterpret_cast<float*>(z), info);
    }
}

struct BatchGuard {
    reform_batch* b;
    ~BatchGuard() { reform_batch_destroy(b); }
};

// The reference's batch call (jrp/pria-cuda/src/pria.cu:15-44 fans independent
// solves out over host threads and streams) as one batched engine
// (include/reform.h): every instance in the same graph replays, each result
// bitwise its solo solve.  The engine runs the restarted Halpern method; plain
// PDHG or a vanilla warm phase falls back to solo solves one after another.
template <class T>
static int solve_batch_engine(int64_t count, int64_t n, int64_t t, const T* k, const T* k0, const T* h,
                              const pria_params* params, T* x, T* y, T* z, pria_result_info* infos) {
    const int64_t full = n * t * t;
    reform_batch* b = nullptr;
    int st = reform_batch_create(sizeof(T) == 4 ? 1 : 0, nullptr, &b);
    if (st) return st < 0 ? -st : st;
    const BatchGuard guard{b};
    std::vector<int> slot;
    for (int64_t i = 0; i < count; ++i) {
        const std::vector<double> costs(k + i * n, k + (i + 1) * n);
        const std::vector<double> holding(h + i * full, h + (i + 1) * full);
        const int id = reform_batch_add_jrp(b, n, t, costs.data(), double(k0[i]), holding.data(), params);
        if (id < 0) return -id;
        slot.push_back(id);
    }
    if ((st = reform_batch_start(b)) || (st = reform_batch_run(b, -1))) return st < 0 ? -st : st;
    std::vector<double> xd, yd, zd;
    if (x) xd.resize(size_t(full));
    if (y) yd.resize(size_t(full));
    if (z) zd.resize(size_t(full));
    for (int64_t i = 0; i < count; ++i) {
        st = reform_batch_result_jrp(b, slot[size_t(i)], x ? xd.data() : nullptr, y ? yd.data() : nullptr,
                                     z ? zd.data() : nullptr, infos ? infos + i : nullptr);
        if (st) return st < 0 ? -st : st;
        for (int64_t a = 0; a < full; ++a) {
            if (x) x[i * full + a] = T(xd[size_t(a)]);
            if (y) y[i * full + a] = T(yd[size_t(a)]);
            if (z) z[i * full + a] = T(zd[size_t(a)]);
        }
    }
    return 0;
}

template <class T>
static int solve_batch(int64_t count, int64_t n, int64_t t, const T* k, const T* k0, const T* h,
                       const pria_params* params, T* x, T* y, T* z, pria_result_info* infos) {
    if (count <= 0 || !k || !k0 || !h || !params) return int(cudaErrorInvalidValue);
    if (n < 1 || t < 1) return int(cudaErrorInvalidValue);
    if (params->use_halpern && params->warm_steps <= 0)
        return solve_batch_engine<T>(count, n, t, k, k0, h, params, x, y, z, infos);
    const int64_t full = n * t * t;
    int err = 0;
    for (int64_t b = 0; b < count; ++b) {
        const int st = solve_one<T>(n, t, k + b * n, k0[b], h + b * full, params, nullptr, nullptr, nullptr,
                                    x ? x + b * full : nullptr, y ? y + b * full : nullptr,
                                    z ? z + b * full : nullptr, infos ? infos + b : nullptr,
                                    sizeof(T) == 4);
        if (st) err = st;
    }
    return err;
}

}  // namespace

extern "C" {

pria_params pria_params_auto(int64_t max_iter, double tolerance) {
    pria_params p;
    p.omega = 0.10835;
    p.eta = 0.999 / std::sqrt(2.0);
    p.beta_sufficient = std::exp(-1.0);
    p.beta_artificial = 0.2468;
    p.beta_necessary = 0.5706;
    p.theta_initial = 0.81930;
    p.theta_target = 0.42818;
    p.theta_decay = 0.90474;
    p.tolerance = tolerance;
    p.max_iter = max_iter;
    p.use_halpern = 1;
    p.warm_steps = 0;
    p.op_steps = 16;
    p.verbose = 0;
    return p;
}

int reform_pria_create(int64_t n, int64_t t, const double* order_costs, double joint_cost,
                       const double* holding_costs, const pria_params* params, int use_float32,
                       void* stream, reform_pria_solver** out) {
    if (!out) return int(cudaErrorInvalidValue);
    *out = nullptr;
    auto s = std::make_unique<reform_pria_solver>();
    const int st = pria::create<double>(n, t, order_costs, joint_cost, holding_costs, params, use_float32,
                                        static_cast<cudaStream_t>(stream), s->impl);
    if (st) return st;
    *out = s.release();
    return 0;
}

int reform_pria_run(reform_pria_solver* solver) {
    if (!solver || !solver->impl) return int(cudaErrorInvalidValue);
    return solver->impl->run();
}

int reform_pria_set_time_limit(reform_pria_solver* solver, double seconds) {
    if (!solver || !solver->impl) return int(cudaErrorInvalidValue);
    solver->impl->time_limit = seconds;
    return 0;
}

int reform_pria_set_warm(reform_pria_solver* solver, const double* wx, const double* wy, const double* wz) {
    if (!solver || !solver->impl) return int(cudaErrorInvalidValue);
    return solver->impl->set_warm(wx, wy, wz);
}

int reform_pria_result(reform_pria_solver* solver, double* x, double* y, double* z, pria_result_info* info) {
    if (!solver || !solver->impl) return int(cudaErrorInvalidValue);
    return solver->impl->result(x, y, z, info);
}

int reform_pria_run_profiled(reform_pria_solver* solver, double* ms, int64_t* count) {
    if (!solver || !solver->impl || !ms || !count) return int(cudaErrorInvalidValue);
    long long c[9];
    const int st = solver->impl->run_profiled(ms, c);
    for (int q = 0; q < 9; ++q) count[q] = c[q];
    return st;
}

int reform_pria_set_trace(reform_pria_solver* solver, int capacity) {
    if (!solver || !solver->impl) return int(cudaErrorInvalidValue);
    return solver->impl->set_trace(capacity);
}

int reform_pria_trace(reform_pria_solver* solver, reform_trace_record* out, int capacity, int64_t* total) {
    if (!solver || !solver->impl) return int(cudaErrorInvalidValue);
    return solver->impl->get_trace(out, capacity, total);
}

int reform_pria_set_megakernel(reform_pria_solver* solver, int mode, int* active) {
    if (!solver || !solver->impl) return int(cudaErrorInvalidValue);
    return solver->impl->set_megakernel(mode, active);
}

int64_t reform_pria_launches(const reform_pria_solver* solver) {
    return solver && solver->impl ? solver->impl->launches() : 0;
}

void reform_pria_destroy(reform_pria_solver* solver) { delete solver; }

int pria_solve_f64(int64_t n, int64_t t, const double* order_costs, double joint_cost,
                   const double* holding_costs, const pria_params* params, const double* warm_x,
                   const double* warm_y, const double* warm_z, double* x, double* y, double* z,
                   pria_result_info* info) {
    return solve_one<double>(n, t, order_costs, joint_cost, holding_costs, params, warm_x, warm_y, warm_z, x,
                             y, z, info, 0);
}

int pria_solve_f32(int64_t n, int64_t t, const float* order_costs, float joint_cost,
                   const float* holding_costs, const pria_params* params, const float* warm_x,
                   const float* warm_y, const float* warm_z, float* x, float* y, float* z,
                   pria_result_info* info) {
    return solve_one<float>(n, t, order_costs, joint_cost, holding_costs, params, warm_x, warm_y, warm_z, x,
                            y, z, info, 1);
}

int pria_solve_batch_f64(int64_t count, int64_t n, int64_t t, const double* order_costs,
                         const double* joint_costs, const double* holding_costs, const pria_params* params,
                         double* x, double* y, double* z, pria_result_info* infos) {
    return solve_batch<double>(count, n, t, order_costs, joint_costs, holding_costs, params, x, y, z, infos);
}

int pria_solve_batch_f32(int64_t count, int64_t n, int64_t t, const float* order_costs,
                         const float* joint_costs, const float* holding_costs, const pria_params* params,
                         float* x, float* y, float* z, pria_result_info* infos) {
    return solve_batch<float>(count, n, t, order_costs, joint_costs, holding_costs, params, x, y, z, infos);
}

double pria_objective_f64(int64_t n, int64_t t, const double* order_costs, double joint_cost,
                          const double* holding_costs, const double* x) {
    // on the host, in FP64: the maxima run over whole rows (jrp_problem.py:143-161)
    double obj = 0.0;
    for (int64_t i = 0; i < n; ++i)
        for (int64_t s = 0; s < t; ++s) {
            double m = 0.0;
            for (int64_t tt = 0; tt < t; ++tt) m = std::max(m, x[(i * t + s) * t + tt]);
            obj += order_costs[i] * m;
        }
    for (int64_t s = 0; s < t; ++s) {
        double m = 0.0;
        for (int64_t i = 0; i < n; ++i)
            for (int64_t tt = 0; tt < t; ++tt) m = std::max(m, x[(i * t + s) * t + tt]);
        obj += joint_cost * m;
    }
    for (int64_t i = 0; i < n; ++i)
        for (int64_t s = 0; s < t; ++s)
            for (int64_t tt = s; tt < t; ++tt) obj += holding_costs[(i * t + s) * t + tt] * x[(i * t + s) * t + tt];
    return obj;
}

}  // extern "C"
