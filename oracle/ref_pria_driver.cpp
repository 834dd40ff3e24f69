// ref_pria_driver.cpp -- a C entry point over the reference's own CPU PRIA
// (jrp/pria-cuda/tests/ref_impl.hpp, namespace ref), compiled in place from the
// reference tree by oracle/Makefile into oracle/_ref/libpria_ref.so.
//
// TEST INFRASTRUCTURE ONLY: the parity tests use it to pin the PRIA oracle
// restatement, and bench.py's reference arm times it as the reference's CPU
// implementation.  Nothing in the product links it.
#include <cstdint>
#include <cstring>

#include "ref_impl.hpp"   // jrp/pria-cuda/tests/ref_impl.hpp (include path set by the Makefile)

extern "C" {

// Solve with ref::solve (ref_impl.hpp:237-422).  params uses the reference's
// pria_params layout (jrp/pria-cuda/include/pria/pria.h:34-49).  out[0..4) =
// iterations, primal, dual, gap as ref::Result carries them.  x/y/z may be NULL.
int ref_pria_solve(int64_t n, int64_t t, const double* k, double k0, const double* h,
                   const pria_params* params, double* x, double* y, double* z, double* out) {
    ref::Instance inst;
    inst.n = n;
    inst.t = t;
    inst.k.assign(k, k + n);
    inst.k0 = k0;
    inst.h.assign(h, h + n * t * t);
    ref::Result r = ref::solve(inst, *params);
    out[0] = double(r.iterations);
    out[1] = r.primal;
    out[2] = r.dual;
    out[3] = r.gap;
    const size_t bytes = sizeof(double) * size_t(n * t * t);
    if (x) std::memcpy(x, r.x.data(), bytes);
    if (y) std::memcpy(y, r.y.data(), bytes);
    if (z) std::memcpy(z, r.z.data(), bytes);
    return 0;
}

// ref::random_instance (ref_impl.hpp:56-80), for instances shaped like the
// reference's own tests.  k[n], h[n*t*t].
void ref_pria_random_instance(uint64_t seed, int64_t n, int64_t t, double* k, double* k0,
                              double* h) {
    ref::Instance inst = ref::random_instance(seed, n, t);
    std::memcpy(k, inst.k.data(), sizeof(double) * size_t(n));
    *k0 = inst.k0;
    std::memcpy(h, inst.h.data(), sizeof(double) * size_t(n * t * t));
}

}  // extern "C"
