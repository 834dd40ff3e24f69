// Test driver for reformulation_b200/cli/wire_format.hpp (host only).
// tests/test_cli.py compiles it with g++ and drives it:
//
//   wire_format_check qubo <file>            load a QUBO instance, print JSON
//   wire_format_check jrp <file>             load a JRP instance, print JSON
//   wire_format_check record <file> W.. -- R.. -- A..
//                                            write a result record: int64
//                                            words, doubles, one array
//   wire_format_check args <argv...>         parse a command line with the
//                                            JRP tool's flag set, print JSON
#include <cstdio>
#include <string>
#include <vector>

#include "wire_format.hpp"

namespace w = rb200::wire;

template <class T>
static void print_array(const char* key, const std::vector<T>& v) {
    std::printf("\"%s\": [", key);
    for (size_t i = 0; i < v.size(); ++i) {
        if constexpr (std::is_same_v<T, double>)
            std::printf("%s%.17g", i ? ", " : "", v[i]);
        else
            std::printf("%s%lld", i ? ", " : "", (long long)v[i]);
    }
    std::printf("]");
}

static void print_error(const std::string& why) {
    std::printf("{\"ok\": false, \"error\": \"%s\"}\n", why.c_str());
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string cmd = argv[1];
    if (cmd == "qubo" && argc == 3) {
        w::QuboFile q;
        std::string why = w::load(argv[2], q);
        if (!why.empty()) return print_error(why), 0;
        std::printf("{\"ok\": true, \"n\": %lld, \"m\": %lld, ", (long long)q.n, (long long)q.m);
        print_array("diag", q.diag), std::printf(", ");
        print_array("rows", q.rows), std::printf(", ");
        print_array("cols", q.cols), std::printf(", ");
        print_array("vals", q.vals), std::printf("}\n");
        return 0;
    }
    if (cmd == "jrp" && argc == 3) {
        w::JrpFile j;
        std::string why = w::load(argv[2], j);
        if (!why.empty()) return print_error(why), 0;
        std::printf("{\"ok\": true, \"n\": %lld, \"t\": %lld, \"k0\": %.17g, ", (long long)j.n,
                    (long long)j.t, j.k0);
        print_array("k", j.k), std::printf(", ");
        print_array("h", j.h), std::printf("}\n");
        return 0;
    }
    if (cmd == "record" && argc >= 3) {
        std::vector<int64_t> words;
        std::vector<double> reals, arr;
        int part = 0;
        for (int k = 3; k < argc; ++k) {
            std::string a = argv[k];
            if (a == "--") {
                ++part;
                continue;
            }
            if (part == 0) words.push_back(std::stoll(a));
            else if (part == 1) reals.push_back(std::stod(a));
            else arr.push_back(std::stod(a));
        }
        w::Record r;
        for (int64_t v : words) r.word(v);
        for (double v : reals) r.real(v);
        if (!arr.empty()) r.array(arr.data(), arr.size());
        std::string why = r.commit(argv[2]);
        if (!why.empty()) return print_error(why), 0;
        std::printf("{\"ok\": true}\n");
        return 0;
    }
    if (cmd == "args") {
        w::Invocation inv;
        // argv[1] ("args") plays the program name
        std::string why = w::parse(argc - 1, argv + 1, {"f32", "vanilla", "verbose", "solution"}, inv);
        if (!why.empty()) return print_error(why), 0;
        std::printf("{\"ok\": true, \"instance\": \"%s\", \"result\": \"%s\", ", inv.instance.c_str(),
                    inv.result.c_str());
        if (inv.has_tolerance)
            std::printf("\"tolerance\": %.17g, ", inv.tolerance);
        else
            std::printf("\"tolerance\": null, ");
        std::printf("\"max_iter\": %s, \"flags\": [",
                    inv.has_max_iter ? std::to_string(inv.max_iter).c_str() : "null");
        for (size_t i = 0; i < inv.flags.size(); ++i)
            std::printf("%s\"%s\"", i ? ", " : "", inv.flags[i].c_str());
        std::printf("]}\n");
        return 0;
    }
    return 2;
}
