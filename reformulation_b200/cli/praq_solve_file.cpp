// praq_solve_file -- the file-driven PRAQ solve, over this library's C ABI.
//
// Drop-in for the reference's CLI (qubo/praq-cuda/tools/praq_solve_file.cu:1-31),
// which its harness backend (qubo/harness/backends/praq_cuda.py:27-86) runs as
// a subprocess.  The wire formats and the exit codes are that contract, so they
// are the same here; the program itself is this project's.
//
//   instance (little-endian):  i64 magic 0x51415250, i64 n, i64 m,
//                              f64 diag[n], i64 rows[m], i64 cols[m], f64 vals[m]
//   result:                    i64 n, i64 iterations, i64 status,
//                              f64 lower, f64 upper, f64 x[n]
//
//   usage: praq_solve_file <instance> <result> [tol] [max_iter] [f32]
//   exit:  0 converged, 1 iteration limit, 2 usage / unreadable input /
//          unwritable result, 3 the solver failed (no result file is written)
//
// Stdout repeats the result as "key: value" lines, with setup_seconds (file
// read + CUDA context) and solve_seconds (the praq_solve call), which the
// harness parses (praq_cuda.py:_timings).
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_runtime_api.h>

#include "praq.h"

namespace {

constexpr int64_t kMagic = 0x51415250;   // "PRAQ"

using Clock = std::chrono::steady_clock;

double since(Clock::time_point t0) {
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

// Reads `count` items of T; false on a short file.
template <class T>
bool read_items(FILE* f, std::vector<T>& v, int64_t count) {
    if (count < 0) return false;
    v.resize(size_t(count));
    return count == 0 || std::fread(v.data(), sizeof(T), size_t(count), f) == size_t(count);
}

struct FileCloser {
    FILE* f;
    ~FileCloser() { if (f) std::fclose(f); }
};

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3 || argc > 6) {
        std::fprintf(stderr, "usage: %s <instance> <result> [tol] [max_iter] [f32]\n", argv[0]);
        return 2;
    }
    PraqParameters params = praq_default_parameters();
    if (argc > 3) params.tolerance = std::atof(argv[3]);
    if (argc > 4) params.max_iter = std::atoll(argv[4]);
    if (argc > 5) params.use_float32 = std::strcmp(argv[5], "f32") == 0 ? 1 : 0;

    const auto t_setup = Clock::now();
    std::vector<double> diag, vals;
    std::vector<int64_t> rows, cols;
    int64_t head[3] = {0, 0, 0};
    {
        FileCloser in{std::fopen(argv[1], "rb")};
        if (!in.f) {
            std::fprintf(stderr, "praq_solve_file: cannot open %s\n", argv[1]);
            return 2;
        }
        const bool ok = std::fread(head, sizeof(int64_t), 3, in.f) == 3 && head[0] == kMagic &&
                        head[1] >= 0 && head[2] >= 0 && read_items(in.f, diag, head[1]) &&
                        read_items(in.f, rows, head[2]) && read_items(in.f, cols, head[2]) &&
                        read_items(in.f, vals, head[2]);
        if (!ok) {
            std::fprintf(stderr, "praq_solve_file: %s is not a PRAQ instance file\n", argv[1]);
            return 2;
        }
    }
    PraqInstance inst;
    inst.n = head[1];
    inst.m = head[2];
    inst.diag = diag.data();
    inst.rows = rows.data();
    inst.cols = cols.data();
    inst.vals = vals.data();

    cudaFree(nullptr);   // context creation belongs to set-up, not to the solve
    const double setup_seconds = since(t_setup);

    std::vector<double> x(size_t(inst.n));
    PraqResult res;
    const auto t_solve = Clock::now();
    const int rc = praq_solve(&inst, &params, x.data(), &res);
    const double solve_seconds = since(t_solve);
    if (rc < 0) {
        std::fprintf(stderr, "praq_solve_file: praq_solve failed with status %d\n", rc);
        return 3;
    }

    {
        FileCloser out{std::fopen(argv[2], "wb")};
        if (!out.f) {
            std::fprintf(stderr, "praq_solve_file: cannot write %s\n", argv[2]);
            return 2;
        }
        const int64_t words[3] = {inst.n, res.iterations, int64_t(res.status)};
        const double bounds[2] = {res.lower, res.upper};
        bool ok = std::fwrite(words, sizeof(int64_t), 3, out.f) == 3 &&
                  std::fwrite(bounds, sizeof(double), 2, out.f) == 2 &&
                  std::fwrite(x.data(), sizeof(double), x.size(), out.f) == x.size();
        ok = std::fclose(out.f) == 0 && ok;
        out.f = nullptr;
        if (!ok) {
            std::fprintf(stderr, "praq_solve_file: short write to %s\n", argv[2]);
            return 2;
        }
    }

    std::printf("n: %lld\n", (long long)inst.n);
    std::printf("edges: %lld\n", (long long)inst.m);
    std::printf("precision: %s\n", params.use_float32 ? "float32" : "float64");
    std::printf("status: %s\n", res.status == 0 ? "converged" : "iteration_limit");
    std::printf("iterations: %lld\n", (long long)res.iterations);
    std::printf("lower: %.17g\n", res.lower);
    std::printf("upper: %.17g\n", res.upper);
    std::printf("setup_seconds: %.6f\n", setup_seconds);
    std::printf("solve_seconds: %.6f\n", solve_seconds);
    return res.status == 0 ? 0 : 1;
}
