// pria_solve_file -- the joint replenishment LP solver as a file-in, file-out
// program, for harnesses that run a solver as a subprocess
// (jrp/harness/backends/pria_cuda.py:83-173 drives it this way).
//
//   pria_solve_file <instance> <result> [tol] [max_iter] [flag ...]
//
//   tol       relative duality gap to stop at (default 1e-4)
//   max_iter  iteration cap; -1 or absent for none
//   flags     f32       FP32 iterates with FP64 reductions and bounds
//             vanilla   plain PDHG instead of the restarted Halpern method
//             verbose   one progress line per check on stderr
//             solution  append x, y, z (normalised duals) to the result file
//
// The file formats, exit codes and the two timing keys are those of
// wire_format.hpp.  The library's result carries bounds and a gap but no
// status word; the status written here is 0 when the gap reached the
// tolerance and 1 otherwise.  The solve uses the device-resident API of
// include/pria.h (set-up, run, result), which takes FP64 input in both
// precisions and converts on the device.
#include <cuda_runtime.h>

#include "pria.h"
#include "wire_format.hpp"

namespace {

constexpr const char* kTool = "pria_solve_file";
constexpr double kDefaultTolerance = 1e-4;
constexpr const char* kUsage =
    "usage: pria_solve_file <instance> <result> [tol] [max_iter] [f32] [vanilla] [verbose] "
    "[solution]";

// Owns a reform_pria_solver for the length of one solve.
struct Solver {
    reform_pria_solver* handle = nullptr;
    ~Solver() {
        if (handle) reform_pria_destroy(handle);
    }
};

}  // namespace

int main(int argc, char** argv) {
    namespace w = rb200::wire;
    const w::Stopwatch setup_clock;

    w::Invocation args;
    if (std::string why = w::parse(argc, argv, {"f32", "vanilla", "verbose", "solution"}, args);
        !why.empty())
        return w::fail(w::kBadInput, kTool, why + "\n" + kUsage);

    w::JrpFile jrp;
    if (std::string why = w::load(args.instance, jrp); !why.empty())
        return w::fail(w::kBadInput, kTool, args.instance + ": " + why);

    pria_params params = pria_params_auto(args.has_max_iter ? args.max_iter : -1,
                                          args.has_tolerance ? args.tolerance : kDefaultTolerance);
    params.use_halpern = args.flag("vanilla") ? 0 : 1;
    params.verbose = args.flag("verbose") ? 1 : 0;
    const bool fp32 = args.flag("f32");
    const bool solution = args.flag("solution");

    if (cudaInitDevice(0, 0, 0) != cudaSuccess || cudaSetDevice(0) != cudaSuccess)
        return w::fail(w::kSolverFailed, kTool, "no usable CUDA device");
    const double setup_seconds = setup_clock.seconds();

    const size_t cells = size_t(jrp.n) * size_t(jrp.t) * size_t(jrp.t);
    std::vector<double> x, y, z;
    if (solution) {
        x.resize(cells);
        y.resize(cells);
        z.resize(cells);
    }
    pria_result_info info{};
    const w::Stopwatch solve_clock;
    Solver solver;
    int err = reform_pria_create(jrp.n, jrp.t, jrp.k.data(), jrp.k0, jrp.h.data(), &params,
                                 fp32 ? 1 : 0, nullptr, &solver.handle);
    if (!err) err = reform_pria_run(solver.handle);
    if (!err)
        err = reform_pria_result(solver.handle, solution ? x.data() : nullptr,
                                 solution ? y.data() : nullptr, solution ? z.data() : nullptr, &info);
    const double solve_seconds = solve_clock.seconds();
    if (err)
        return w::fail(w::kSolverFailed, kTool,
                       std::string("solve failed: ") + cudaGetErrorString(cudaError_t(err)));

    // NaN never counts as converged.
    const int64_t status = info.relative_gap <= params.tolerance ? 0 : 1;
    w::Record record;
    record.word(jrp.n).word(jrp.t).word(info.iterations).word(status);
    record.real(info.dual_objective).real(info.primal_objective).real(info.relative_gap);
    if (solution) record.array(x.data(), cells).array(y.data(), cells).array(z.data(), cells);
    if (std::string why = record.commit(args.result); !why.empty())
        return w::fail(w::kSolverFailed, kTool, why);

    w::Report()
        .add("instance", args.instance)
        .add("items", jrp.n)
        .add("periods", jrp.t)
        .add("precision", std::string(fp32 ? "float32" : "float64"))
        .add("method", std::string(params.use_halpern ? "halpern" : "vanilla"))
        .add("tolerance", params.tolerance)
        .add("status", std::string(status == 0 ? "converged" : "iteration_limit"))
        .add("iterations", info.iterations)
        .add("lower", info.dual_objective)
        .add("upper", info.primal_objective)
        .add("relative_gap", info.relative_gap)
        .add("setup_seconds", setup_seconds)
        .add("solve_seconds", solve_seconds)
        .print();
    return status == 0 ? w::kConverged : w::kIterationLimit;
}
