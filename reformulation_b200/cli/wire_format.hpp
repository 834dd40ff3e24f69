// wire_format.hpp -- the file contract between the solver CLIs and the
// harness that drives them as subprocesses.
//
// The formats are fixed by the reference's harness backends, which write the
// instance file, run the CLI and parse the result file and the stdout timing
// lines (qubo/harness/backends/praq_cuda.py:27-77 and
// jrp/harness/backends/pria_cuda.py:30-78; contract comments at
// qubo/praq-cuda/tools/praq_solve_file.cu:7-31 and
// jrp/pria-cuda/tools/pria_solve_file.cu:7-45).  Everything is little-endian:
//
//   QUBO instance   i64 magic 0x51415250 ("PRAQ"), i64 n, i64 m,
//                   f64 diag[n], i64 rows[m], i64 cols[m], f64 vals[m]
//   QUBO result     i64 n, i64 iterations, i64 status, f64 lower, f64 upper,
//                   f64 x[n]
//   JRP instance    i64 magic 0x41495250 ("PRIA"), i64 n, i64 t, f64 k0,
//                   f64 k[n], f64 h[n*t*t]
//   JRP result      i64 n, i64 t, i64 iterations, i64 status, f64 lower,
//                   f64 upper, f64 gap [, f64 x, y, z each n*t*t]
//
// Exit status: 0 converged, 1 iteration limit, 2 usage error or unreadable
// input, 3 the solver failed.  The result file exists only after a solve
// that ran; this module writes it under a temporary name and renames it into
// place, so a reader never sees a partial record.  Stdout carries
// "key: value" lines, among them setup_seconds (reading the input and creating
// the CUDA context) and solve_seconds (the solve call), the two the harness
// reads.
//
// Host C++17 only; no CUDA types, so the module is unit-tested on its own
// (tests/wire_format_check.cpp).
#pragma once

#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <utility>
#include <vector>

#if !defined(__BYTE_ORDER__) || __BYTE_ORDER__ != __ORDER_LITTLE_ENDIAN__
#error "the wire formats are little-endian; this module reads and writes host order"
#endif

namespace rb200::wire {

constexpr int64_t kQuboMagic = 0x51415250;   // "PRAQ" read as a little-endian word
constexpr int64_t kJrpMagic = 0x41495250;    // "PRIA"

enum Exit : int { kConverged = 0, kIterationLimit = 1, kBadInput = 2, kSolverFailed = 3 };

// ---- reading --------------------------------------------------------------

// A binary file read front to back with typed, size-checked reads.  The total
// size is known up front, so a header's claimed payload can be checked against
// it before anything is allocated.
class Source {
  public:
    explicit Source(const std::string& path) : file_(std::fopen(path.c_str(), "rb")) {
        if (!file_) {
            error_ = "cannot open " + path + ": " + std::strerror(errno);
            return;
        }
        if (std::fseek(file_, 0, SEEK_END) != 0 || (size_ = std::ftell(file_)) < 0 ||
            std::fseek(file_, 0, SEEK_SET) != 0) {
            error_ = "cannot size " + path;
            size_ = 0;
        }
    }
    ~Source() {
        if (file_) std::fclose(file_);
    }
    Source(const Source&) = delete;
    Source& operator=(const Source&) = delete;

    bool ok() const { return error_.empty(); }
    const std::string& error() const { return error_; }
    int64_t unread() const { return size_ - offset_; }

    template <class T>
    bool take(T* into, int64_t count) {
        if (!ok()) return false;
        if (count < 0 || count > unread() / int64_t(sizeof(T))) {
            error_ = "file ends early";
            return false;
        }
        size_t got = count ? std::fread(into, sizeof(T), size_t(count), file_) : 0;
        if (got != size_t(count)) {
            error_ = "read failed";
            return false;
        }
        offset_ += count * int64_t(sizeof(T));
        return true;
    }
    template <class T>
    bool take(std::vector<T>& into, int64_t count) {
        if (count < 0 || count > unread() / int64_t(sizeof(T))) {
            error_ = "file ends early";
            return false;
        }
        into.resize(size_t(count));
        return take(into.data(), count);
    }

  private:
    std::FILE* file_ = nullptr;
    int64_t size_ = 0;
    int64_t offset_ = 0;
    std::string error_;
};

// Payload bytes of `words` int64s and `reals` doubles, or -1 on overflow.
inline int64_t payload(int64_t int_words, int64_t real_words) {
    constexpr int64_t kMax = std::numeric_limits<int64_t>::max() / 8;
    if (int_words < 0 || real_words < 0 || int_words > kMax - real_words) return -1;
    return 8 * (int_words + real_words);
}

struct QuboFile {
    int64_t n = 0, m = 0;
    std::vector<double> diag, vals;
    std::vector<int64_t> rows, cols;
};

struct JrpFile {
    int64_t n = 0, t = 0;
    double k0 = 0.0;
    std::vector<double> k, h;
};

// Both loaders return "" on success or a one-line reason.  A file is accepted
// only when its size is exactly what its header announces.
inline std::string load(const std::string& path, QuboFile& q) {
    Source src(path);
    int64_t head[3];
    if (!src.take(head, 3)) return src.error();
    if (head[0] != kQuboMagic) return "wrong magic word: not a QUBO (PRAQ) instance file";
    q.n = head[1];
    q.m = head[2];
    if (q.n <= 0 || q.m < 0) return "bad header: need n > 0 and m >= 0";
    int64_t need = q.m <= std::numeric_limits<int64_t>::max() / 3 ? payload(2 * q.m, q.n + q.m) : -1;
    if (need < 0 || need != src.unread())
        return "size mismatch: the header's n and m do not match the file length";
    if (!src.take(q.diag, q.n) || !src.take(q.rows, q.m) || !src.take(q.cols, q.m) ||
        !src.take(q.vals, q.m))
        return src.error();
    return "";
}

inline std::string load(const std::string& path, JrpFile& j) {
    Source src(path);
    int64_t head[3];
    if (!src.take(head, 3)) return src.error();
    if (head[0] != kJrpMagic) return "wrong magic word: not a JRP (PRIA) instance file";
    j.n = head[1];
    j.t = head[2];
    if (j.n <= 0 || j.t <= 0) return "bad header: need n > 0 and t > 0";
    constexpr int64_t kMax = std::numeric_limits<int64_t>::max() / 8;
    bool fits = j.t <= kMax / j.t && j.n <= kMax / (j.t * j.t);
    int64_t need = fits ? payload(0, 1 + j.n + j.n * j.t * j.t) : -1;
    if (need < 0 || need != src.unread())
        return "size mismatch: the header's n and t do not match the file length";
    if (!src.take(&j.k0, 1) || !src.take(j.k, j.n) || !src.take(j.h, j.n * j.t * j.t))
        return src.error();
    return "";
}

// ---- writing --------------------------------------------------------------

// A result record: int64 words, then doubles, then optional double arrays.
class Record {
  public:
    Record& word(int64_t v) {
        words_.push_back(v);
        return *this;
    }
    Record& real(double v) {
        reals_.push_back(v);
        return *this;
    }
    Record& array(const double* data, size_t count) {
        arrays_.emplace_back(data, count);
        return *this;
    }

    // Write to "<path>.partial" and rename over `path`.  Returns "" or a reason.
    std::string commit(const std::string& path) const {
        const std::string tmp = path + ".partial";
        std::FILE* f = std::fopen(tmp.c_str(), "wb");
        if (!f) return "cannot create " + tmp + ": " + std::strerror(errno);
        bool ok = put(f, words_.data(), words_.size()) && put(f, reals_.data(), reals_.size());
        for (const auto& a : arrays_) ok = ok && put(f, a.first, a.second);
        ok = (std::fclose(f) == 0) && ok;
        if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) {
            std::remove(tmp.c_str());
            return "cannot write " + path;
        }
        return "";
    }

  private:
    template <class T>
    static bool put(std::FILE* f, const T* p, size_t count) {
        return count == 0 || std::fwrite(p, sizeof(T), count, f) == count;
    }
    std::vector<int64_t> words_;
    std::vector<double> reals_;
    std::vector<std::pair<const double*, size_t>> arrays_;
};

// ---- the command line -----------------------------------------------------

// <instance> <result> [tol] [max_iter] [flag ...]: two paths, then up to two
// numbers in that order, then words from the tool's own flag set.
struct Invocation {
    std::string instance, result;
    bool has_tolerance = false, has_max_iter = false;
    double tolerance = 0.0;
    int64_t max_iter = 0;
    std::vector<std::string> flags;

    bool flag(const char* name) const {
        for (const auto& f : flags)
            if (f == name) return true;
        return false;
    }
};

inline bool parse_real(const char* s, double& out) {
    char* end = nullptr;
    errno = 0;
    out = std::strtod(s, &end);
    return end != s && *end == '\0' && errno == 0 && std::isfinite(out);
}

inline bool parse_int(const char* s, int64_t& out) {
    char* end = nullptr;
    errno = 0;
    long long v = std::strtoll(s, &end, 10);
    out = v;
    return end != s && *end == '\0' && errno == 0;
}

// Returns "" or what is wrong with the arguments.
inline std::string parse(int argc, char** argv, const std::vector<std::string>& known_flags,
                         Invocation& inv) {
    if (argc < 3) return "missing the instance and result paths";
    inv.instance = argv[1];
    inv.result = argv[2];
    int k = 3;
    if (k < argc && parse_real(argv[k], inv.tolerance)) {
        if (!(inv.tolerance > 0.0)) return "the tolerance must be positive";
        inv.has_tolerance = true;
        ++k;
        if (k < argc && parse_int(argv[k], inv.max_iter)) {
            inv.has_max_iter = true;
            ++k;
        }
    }
    for (; k < argc; ++k) {
        bool known = false;
        for (const auto& f : known_flags) known = known || f == argv[k];
        if (!known) return std::string("unexpected argument '") + argv[k] + "'";
        inv.flags.push_back(argv[k]);
    }
    return "";
}

// ---- stdout ---------------------------------------------------------------

class Report {
  public:
    Report& add(const char* key, const std::string& value) {
        lines_.emplace_back(key, value);
        return *this;
    }
    Report& add(const char* key, int64_t value) { return add(key, std::to_string(value)); }
    Report& add(const char* key, double value) {
        char buf[64];
        std::snprintf(buf, sizeof buf, "%.17g", value);
        return add(key, std::string(buf));
    }
    void print(std::FILE* out = stdout) const {
        for (const auto& kv : lines_) std::fprintf(out, "%s: %s\n", kv.first, kv.second.c_str());
        std::fflush(out);
    }

  private:
    std::vector<std::pair<const char*, std::string>> lines_;
};

class Stopwatch {
  public:
    double seconds() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - start_).count();
    }

  private:
    std::chrono::steady_clock::time_point start_ = std::chrono::steady_clock::now();
};

// A failure before or around the solve: one line on stderr and the exit code.
inline int fail(Exit code, const char* tool, const std::string& why) {
    std::fprintf(stderr, "%s: %s\n", tool, why.c_str());
    return code;
}

}  // namespace rb200::wire
