// praq_solver.cu -- the C ABI of the PRAQ solver (include/praq.h); the
// solver itself (kernels, device layout, host driver) is praq_core.cuh.
#include "praq_core.cuh"

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
    (void)cudaGetLastError();   // a stale error of an unrelated earlier call is not ours
    PraqParameters p = *parameters;
    if (!praq::valid(p)) return PRAQ_ERROR_ARGUMENT;
    // The reference's limits (qubo/praq-cuda/src/solver.cuh:525-526): node
    // and edge ids are int32 on the device.
    const int64_t limit = std::numeric_limits<int>::max();
    if (instance->n <= 0 || instance->n > limit || instance->m < 0 || instance->m > limit / 2)
        return PRAQ_ERROR_INSTANCE;
    if (!instance->diag || (instance->m > 0 && (!instance->rows || !instance->cols || !instance->vals)))
        return PRAQ_ERROR_INSTANCE;
    if (p.max_iter <= 0) p.max_iter = -1;
    if (p.op_steps <= 0) p.op_steps = praq_check_interval(instance->n, &p);
    if (p.op_steps < 2) p.op_steps = 2;
    auto solver = std::make_unique<reform_praq_solver>();
    auto make = [&](auto* impl) -> int {
        impl->p = p;
        solver->impl.reset(impl);
        return impl->setup(*instance, static_cast<cudaStream_t>(stream));
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

int reform_praq_set_warm(reform_praq_solver* solver, const double* x, const double* y2) {
    if (!solver || !solver->impl) return PRAQ_ERROR_ARGUMENT;
    return solver->impl->set_warm(x, y2);
}

int reform_praq_set_time_limit(reform_praq_solver* solver, double seconds) {
    if (!solver || !solver->impl) return PRAQ_ERROR_ARGUMENT;
    solver->impl->time_limit = seconds;
    return 0;
}

int reform_praq_run_profiled(reform_praq_solver* solver, double* ms, int64_t* count) {
    if (!solver || !solver->impl || !ms || !count) return PRAQ_ERROR_ARGUMENT;
    long long c[10];
    const int st = solver->impl->run_profiled(ms, c);
    for (int k = 0; k < 10; ++k) count[k] = c[k];
    return st;
}

int reform_praq_set_trace(reform_praq_solver* solver, int capacity) {
    if (!solver || !solver->impl) return PRAQ_ERROR_ARGUMENT;
    return solver->impl->set_trace(capacity);
}

int reform_praq_trace(reform_praq_solver* solver, reform_trace_record* out, int capacity, int64_t* total) {
    if (!solver || !solver->impl) return PRAQ_ERROR_ARGUMENT;
    return solver->impl->get_trace(out, capacity, total);
}

int reform_praq_set_megakernel(reform_praq_solver* solver, int mode, int* active) {
    if (!solver || !solver->impl) return PRAQ_ERROR_ARGUMENT;
    return solver->impl->set_megakernel(mode, active);
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
