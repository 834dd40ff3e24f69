// pria_solve_file -- the file-driven PRIA solve, over this library's C ABI.
//
// Drop-in for the reference's CLI (jrp/pria-cuda/tools/pria_solve_file.cu:1-45),
// which its harness backend (jrp/harness/backends/pria_cuda.py) runs as a
// subprocess.  The wire formats, flags and exit codes are that contract, so
// they are the same here; the program itself is this project's.
//
//   instance (little-endian):  i64 magic 0x41495250, i64 n, i64 t, f64 k0,
//                              f64 k[n], f64 h[n t t] (row-major, s <= t read)
//   result:                    i64 n, i64 t, i64 iterations, i64 status,
//                              f64 lower, f64 upper, f64 gap
//                              [f64 x[n t t], y[n t t], z[n t t] with `solution`]
//
//   usage: pria_solve_file <instance> <result> [tol] [max_iter] [flag...]
//          flags: f32 (FP32 iterates), vanilla (plain PDHG), verbose
//          (per-check progress on stderr), solution (write x, y, z)
//   exit:  0 converged, 1 iteration limit, 2 usage / unreadable input /
//          unwritable result, 3 the solver failed (no result file is written)
//
// The library's pria_result_info has no status; as in the reference, it is
// derived here from whether the gap reached the requested tolerance.  lower is
// the dual objective, upper the primal objective at the returned x.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_runtime_api.h>

#include "pria.h"

namespace {

constexpr int64_t kMagic = 0x41495250;   // "PRIA"

using Clock = std::chrono::steady_clock;

double since(Clock::time_point t0) {
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

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
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s <instance> <result> [tol] [max_iter] [f32|vanilla|verbose|solution]...\n",
                     argv[0]);
        return 2;
    }
    const double tol = argc > 3 ? std::atof(argv[3]) : 1e-4;
    const int64_t max_iter = argc > 4 ? std::atoll(argv[4]) : -1;
    bool f32 = false, vanilla = false, verbose = false, solution = false;
    for (int a = 5; a < argc; ++a) {
        if (!std::strcmp(argv[a], "f32")) f32 = true;
        else if (!std::strcmp(argv[a], "vanilla")) vanilla = true;
        else if (!std::strcmp(argv[a], "verbose")) verbose = true;
        else if (!std::strcmp(argv[a], "solution")) solution = true;
        else {
            std::fprintf(stderr, "pria_solve_file: unknown flag %s\n", argv[a]);
            return 2;
        }
    }

    const auto t_setup = Clock::now();
    int64_t head[3] = {0, 0, 0};
    double k0 = 0.0;
    std::vector<double> k, h;
    {
        FileCloser in{std::fopen(argv[1], "rb")};
        if (!in.f) {
            std::fprintf(stderr, "pria_solve_file: cannot open %s\n", argv[1]);
            return 2;
        }
        bool ok = std::fread(head, sizeof(int64_t), 3, in.f) == 3 && head[0] == kMagic && head[1] > 0 &&
                  head[2] > 0 && std::fread(&k0, sizeof(double), 1, in.f) == 1 &&
                  read_items(in.f, k, head[1]);
        // n t^2 must not overflow before the read is attempted
        ok = ok && head[2] <= (int64_t(1) << 20) && head[1] <= (int64_t(1) << 62) / (head[2] * head[2]) &&
             read_items(in.f, h, head[1] * head[2] * head[2]);
        if (!ok) {
            std::fprintf(stderr, "pria_solve_file: %s is not a PRIA instance file\n", argv[1]);
            return 2;
        }
    }
    const int64_t n = head[1], t = head[2];
    const size_t size = size_t(n) * size_t(t) * size_t(t);

    pria_params params = pria_params_auto(max_iter, tol);
    params.use_halpern = vanilla ? 0 : 1;
    params.verbose = verbose ? 1 : 0;

    cudaFree(nullptr);   // context creation belongs to set-up, not to the solve
    const double setup_seconds = since(t_setup);

    std::vector<double> x, y, z;
    if (solution) {
        x.resize(size);
        y.resize(size);
        z.resize(size);
    }
    pria_result_info info;
    int rc;
    const auto t_solve = Clock::now();
    if (f32) {
        std::vector<float> kf(k.begin(), k.end()), hf(h.begin(), h.end());
        std::vector<float> xf, yf, zf;
        if (solution) {
            xf.resize(size);
            yf.resize(size);
            zf.resize(size);
        }
        rc = pria_solve_f32(n, t, kf.data(), float(k0), hf.data(), &params, nullptr, nullptr, nullptr,
                            solution ? xf.data() : nullptr, solution ? yf.data() : nullptr,
                            solution ? zf.data() : nullptr, &info);
        for (size_t g = 0; solution && g < size; ++g) {
            x[g] = xf[g];
            y[g] = yf[g];
            z[g] = zf[g];
        }
    } else {
        rc = pria_solve_f64(n, t, k.data(), k0, h.data(), &params, nullptr, nullptr, nullptr,
                            solution ? x.data() : nullptr, solution ? y.data() : nullptr,
                            solution ? z.data() : nullptr, &info);
    }
    const double solve_seconds = since(t_solve);
    if (rc != 0) {
        std::fprintf(stderr, "pria_solve_file: pria_solve failed with status %d\n", rc);
        return 3;
    }

    const double lower = info.dual_objective, upper = info.primal_objective;
    const int64_t status = std::isfinite(info.relative_gap) && info.relative_gap <= tol ? 0 : 1;
    {
        FileCloser out{std::fopen(argv[2], "wb")};
        if (!out.f) {
            std::fprintf(stderr, "pria_solve_file: cannot write %s\n", argv[2]);
            return 2;
        }
        const int64_t words[4] = {n, t, info.iterations, status};
        const double bounds[3] = {lower, upper, info.relative_gap};
        bool ok = std::fwrite(words, sizeof(int64_t), 4, out.f) == 4 &&
                  std::fwrite(bounds, sizeof(double), 3, out.f) == 3;
        if (ok && solution)
            ok = std::fwrite(x.data(), sizeof(double), size, out.f) == size &&
                 std::fwrite(y.data(), sizeof(double), size, out.f) == size &&
                 std::fwrite(z.data(), sizeof(double), size, out.f) == size;
        ok = std::fclose(out.f) == 0 && ok;
        out.f = nullptr;
        if (!ok) {
            std::fprintf(stderr, "pria_solve_file: short write to %s\n", argv[2]);
            return 2;
        }
    }

    std::printf("items: %lld\n", (long long)n);
    std::printf("periods: %lld\n", (long long)t);
    std::printf("precision: %s\n", f32 ? "float32" : "float64");
    std::printf("status: %s\n", status == 0 ? "converged" : "iteration_limit");
    std::printf("iterations: %lld\n", (long long)info.iterations);
    std::printf("lower: %.17g\n", lower);
    std::printf("upper: %.17g\n", upper);
    std::printf("relative_gap: %.6e\n", info.relative_gap);
    std::printf("setup_seconds: %.6f\n", setup_seconds);
    std::printf("solve_seconds: %.6f\n", solve_seconds);
    return int(status);
}
