// praq_solve_file -- the QUBO roof-dual LP solver as a file-in, file-out
// program, for harnesses that run a solver as a subprocess
// (qubo/harness/backends/praq_cuda.py:79-167 drives it this way).
//
//   praq_solve_file <instance> <result> [tol] [max_iter] [f32]
//
//   tol       relative duality gap to stop at (default: the library's)
//   max_iter  iteration cap; 0 or absent keeps the library's default
//   f32       FP32 iterates with FP64 reductions and bounds
//
// The file formats, exit codes and the two timing keys are those of
// wire_format.hpp.  The solve goes through praq_solve, the reference-facing
// entry point of include/praq.h.
#include <cuda_runtime.h>

#include "praq.h"
#include "wire_format.hpp"

namespace {

constexpr const char* kTool = "praq_solve_file";
constexpr const char* kUsage =
    "usage: praq_solve_file <instance> <result> [tol] [max_iter] [f32]";

const char* status_name(int status) {
    switch (status) {
        case 0: return "converged";
        case 1: return "iteration_limit";
        default: return "error";
    }
}

}  // namespace

int main(int argc, char** argv) {
    namespace w = rb200::wire;
    const w::Stopwatch setup_clock;

    w::Invocation args;
    if (std::string why = w::parse(argc, argv, {"f32"}, args); !why.empty())
        return w::fail(w::kBadInput, kTool, why + "\n" + kUsage);

    w::QuboFile qubo;
    if (std::string why = w::load(args.instance, qubo); !why.empty())
        return w::fail(w::kBadInput, kTool, args.instance + ": " + why);

    PraqParameters params = praq_default_parameters();
    if (args.has_tolerance) params.tolerance = args.tolerance;
    if (args.has_max_iter && args.max_iter != 0) params.max_iter = args.max_iter;
    params.use_float32 = args.flag("f32") ? 1 : 0;

    // The CUDA context belongs to set-up, not to the solve.
    if (cudaInitDevice(0, 0, 0) != cudaSuccess || cudaSetDevice(0) != cudaSuccess)
        return w::fail(w::kSolverFailed, kTool, "no usable CUDA device");
    const double setup_seconds = setup_clock.seconds();

    const PraqInstance view{qubo.n, qubo.m, qubo.diag.data(), qubo.rows.data(), qubo.cols.data(),
                            qubo.vals.data()};
    std::vector<double> x(size_t(qubo.n));
    PraqResult result{};
    const w::Stopwatch solve_clock;
    const int status = praq_solve(&view, &params, x.data(), &result);
    const double solve_seconds = solve_clock.seconds();
    if (status < 0)
        return w::fail(w::kSolverFailed, kTool,
                       "praq_solve returned error " + std::to_string(status));

    w::Record record;
    record.word(qubo.n).word(result.iterations).word(status);
    record.real(result.lower).real(result.upper);
    record.array(x.data(), x.size());
    if (std::string why = record.commit(args.result); !why.empty())
        return w::fail(w::kSolverFailed, kTool, why);

    const double gap =
        (result.upper - result.lower) / (1.0 + std::fabs(result.upper) + std::fabs(result.lower));
    w::Report()
        .add("instance", args.instance)
        .add("nodes", qubo.n)
        .add("edges", qubo.m)
        .add("precision", std::string(params.use_float32 ? "float32" : "float64"))
        .add("tolerance", params.tolerance)
        .add("status", std::string(status_name(status)))
        .add("iterations", result.iterations)
        .add("lower", result.lower)
        .add("upper", result.upper)
        .add("relative_gap", gap)
        .add("setup_seconds", setup_seconds)
        .add("solve_seconds", solve_seconds)
        .print();
    return status == 0 ? w::kConverged : w::kIterationLimit;
}
