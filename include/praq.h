/* praq.h -- C ABI of the B200 PRAQ solver (QUBO roof-dual LP by restarted,
 * reflected Halpern PDHG on the half-edge lift).
 *
 * The first block is a drop-in for the reference's libpraq.so: the same entry
 * points, struct layouts, argument meaning and error codes, so the reference's
 * ctypes `Library` (qubo/harness/praq_cuda_library.py:90-139) and its file CLI
 * contract bind to this library unchanged.
 *
 *   PraqInstance / PraqParameters / PraqResult  replace
 *       qubo/praq-cuda/include/praq/praq.h:20-67 (field for field)
 *   praq_default_parameters   replaces qubo/praq-cuda/include/praq/praq.h:71
 *                             (defaults of Parameters.with_auto_step,
 *                             qubo/praq-jax/praq/solver.py:129-164)
 *   praq_check_interval       replaces qubo/praq-cuda/include/praq/praq.h:76
 *   praq_solve                replaces qubo/praq-cuda/include/praq/praq.h:85-86
 *
 * The second block (reform_praq_*) has no counterpart in the reference: it
 * splits a solve into set-up (validation, device layout, upload) and repeated
 * device-resident solves on a caller-supplied CUDA stream, which is what the
 * batch engine and the timing harness need.
 *
 * All host pointers are caller-owned and only read (outputs only written).
 * Every call is thread-safe: each solve runs on its own stream and device
 * allocations, and touches neither the legacy default stream nor other
 * solves' memory.
 */
#ifndef REFORM_B200_PRAQ_H
#define REFORM_B200_PRAQ_H

#include <stdint.h>

#include "reform_trace.h"

#ifndef REFORM_API
#define REFORM_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* min_{x in {0,1}^n} x^T W x; W symmetric, diagonal + strict upper COO. */
typedef struct {
    int64_t n;              /* binary variables                                 */
    int64_t m;              /* off-diagonal nonzeros (edges), rows[e] != cols[e] */
    const double* diag;     /* [n]                                              */
    const int64_t* rows;    /* [m]                                              */
    const int64_t* cols;    /* [m]                                              */
    const double* vals;     /* [m], W_ij = W_ji                                 */
} PraqInstance;

typedef struct {
    double tolerance;       /* relative duality gap at termination              */
    int64_t max_iter;       /* <= 0: no cap                                     */
    int use_float32;        /* 0: FP64 iterates; 1: FP32 iterates with FP64
                               reductions, restart logic and bounds            */
    double omega;           /* initial primal weight                            */
    double beta_sufficient;
    double beta_necessary;
    double beta_artificial;
    double theta_initial;
    double theta_target;
    double theta_decay;
    int64_t op_steps;       /* iterations between checks (>= 2); <= 0: the rule */
    double interval_offset; /* check-interval rule, see praq_check_interval    */
    double interval_scale;
    double interval_power;
} PraqParameters;

typedef struct {
    double lower;           /* valid lower bound on the relaxation optimum      */
    double upper;           /* relaxation value F(x) at the returned primal     */
    int64_t iterations;
    int status;             /* 0 converged, 1 iteration limit, < 0 error        */
} PraqResult;

/* Error codes (negative), as the reference's. */
#define PRAQ_ERROR_ARGUMENT (-1)   /* null pointer or bad parameter             */
#define PRAQ_ERROR_INSTANCE (-2)   /* index out of range, self-loop, n = 0,
                                      or sizes beyond int32 indexing            */
#define PRAQ_ERROR_CUDA     (-3)   /* any CUDA runtime failure                  */

REFORM_API PraqParameters praq_default_parameters(void);

/* max(2, round(offset + scale * B(ln(n / 50000), power))), B the Box-Cox
 * transform; 2 for a null pointer or n <= 0. */
REFORM_API int64_t praq_check_interval(int64_t n, const PraqParameters* parameters);

/* Solve the roof-dual LP.  x receives the primal [n].  Returns result->status. */
REFORM_API int praq_solve(const PraqInstance* instance, const PraqParameters* parameters,
               double* x, PraqResult* result);

/* ---- device-resident solves (no reference counterpart) ------------------- */

typedef struct reform_praq_solver reform_praq_solver;

/* Validate, lay the instance out on the device and capture the iteration
 * graphs, on `stream` (a cudaStream_t; NULL makes a private non-blocking
 * stream).  Returns 0 or a PRAQ_ERROR_* code. */
REFORM_API int reform_praq_create(const PraqInstance* instance, const PraqParameters* parameters,
                       void* stream, reform_praq_solver** out);

/* One full solve from the cold start on the device-resident instance.  Blocks
 * the host until the solve has finished (the restart/termination decisions are
 * taken on the device; the host only watches a flag).  Returns the status. */
REFORM_API int reform_praq_run(reform_praq_solver* solver);

/* The last run's primal (x may be NULL), dual pairs in instance units
 * (y2 [2m], may be NULL) and result. */
REFORM_API int reform_praq_result(reform_praq_solver* solver, double* x, double* y2, PraqResult* result);

/* A warm start for the following runs, as the reference's
 * solve_qubo_problem_warm_start (qubo/praq-jax/praq/solver.py:482-560): x [n]
 * and dual pairs y2 [2m] in instance units and the instance's own edge order
 * (what reform_praq_result returns); both are projected (x clipped to [0, 1],
 * each pair onto its edge's dual set), so any point may be given.  Either may
 * be NULL (x = 1/2, or the centroid of the dual set); both NULL restores the
 * cold start.  The arrays are copied; the call returns when they are. */
REFORM_API int reform_praq_set_warm(reform_praq_solver* solver, const double* x, const double* y2);

/* A wall-clock budget for each run, in seconds (< 0: none, the default).
 * When it runs out the run stops between two checks and returns
 * PRAQ_STATUS_TIME_LIMIT; the result is the bracket of the last completed
 * check (valid: both iterates stay feasible) and the current primal iterate. */
#define PRAQ_STATUS_TIME_LIMIT 2
REFORM_API int reform_praq_set_time_limit(reform_praq_solver* solver, double seconds);

/* A measurement run: the same solve with every kernel launched on its own
 * between a pair of CUDA events on the solver's stream.  ms[10] and count[10]
 * receive each kernel kind's total device milliseconds and launch count, in
 * this order: node step, edge step, node step with check sums, edge step with
 * check sums, lower-bound pass, check, restart node step, restart edge step,
 * restart check, and a whole check block of the persistent kernel (below).
 * Returns the status like reform_praq_run. */
REFORM_API int reform_praq_run_profiled(reform_praq_solver* solver, double* ms, int64_t* count);

/* Small instances: the persistent kernel, in place of the captured graph of
 * one kernel per phase, in two forms.  The single-CTA form copies the whole
 * instance into one CTA's shared memory (up to about 3,000 edges in FP64,
 * 5,000 in FP32) and runs the start step and up to 128 check blocks per
 * launch there, with block barriers between phases.  The grid form runs one
 * check block per cooperative launch with its phases (node step; edge step;
 * lower bound; check; restart step) separated by grid barriers.  No
 * counterpart in the reference's praq-cuda; its pria-cuda has a megakernel
 * (PRIA_MEGA).  `mode` -1: automatic (the default: the single-CTA form for
 * at most 2,048 edges, where it measured 1.5-2x faster per solve than the
 * graph, else the graph), 0: the graph, 1: the single-CTA form
 * when the instance fits, else the grid form, 2: the grid form.  Both forms
 * need the slot-1 push layout (edge arrays within twice the L2 size).
 * REFORM_PRAQ_MEGA=0|1 in the environment sets the mode at creation.
 * *active (may be NULL) receives the form later runs take: 0 the graph, 1 the
 * grid form, 2 the single-CTA form.  Results equal the graph's bit for bit
 * (the same tile functions, tile shapes and sums).  Every grid-barrier wait is
 * bounded (1 s of device time): one that runs out ends the launch and the run
 * returns PRAQ_ERROR_CUDA with the context still usable. */
REFORM_API int reform_praq_set_megakernel(reform_praq_solver* solver, int mode, int* active);

/* The convergence trace (include/reform_trace.h): later runs write one record
 * per convergence check into a device ring of `capacity` records (0: no
 * trace, the default), from the start of each run.  Setting it drops the
 * solver's captured block (the next run captures a new one).  Returns 0 or
 * PRAQ_ERROR_CUDA. */
REFORM_API int reform_praq_set_trace(reform_praq_solver* solver, int capacity);

/* The last run's trace, oldest first: the most recent min(written, ring
 * capacity, `capacity`) records into `out`; *total (may be NULL) receives the
 * number the run wrote (more than the ring holds when it wrapped). */
REFORM_API int reform_praq_trace(reform_praq_solver* solver, reform_trace_record* out, int capacity,
                                 int64_t* total);

/* Kernel launches the last run issued (graph kernel nodes included). */
REFORM_API int64_t reform_praq_launches(const reform_praq_solver* solver);

REFORM_API void reform_praq_destroy(reform_praq_solver* solver);

/* ---- the bracket of a given point, with no device allocation ------------- */

/* No counterpart in the reference.  The roof-dual bracket of a primal-dual
 * pair, lower = L_D(y) and upper = F(x) in the instance's own units (the
 * reference's relaxation_bounds, qubo/praq-jax/praq/solver.py:348-362), for
 * callers that cannot allocate device memory where they need it: code running
 * inside its own stream capture (allocation is not capturable), real-time
 * loops that must not touch the allocator, and frameworks that own all device
 * memory and hand a library only buffers.
 *
 * Every pointer is DEVICE memory the caller owns: diag [n], rows/cols [m]
 * (int64), vals [m], x [n], y [2m] (half-edge pairs), out [2] = (lower, upper).
 * The work is enqueued on `stream` (a cudaStream_t; NULL = the legacy stream)
 * and is complete when that stream is; the call itself does not synchronise.
 *
 * The scratch is one fixed file-scope device array of 262,144 + 1,185 doubles
 * (about 2 MiB), held by every GPU that loads the library until the process
 * exits.  Limits: 1 <= n <= 262,144 (PRAQ_ERROR_INSTANCE beyond it), any m.
 * The first call on a device looks up the array's device address (with that
 * device current) and caches it: make that first call before any stream
 * capture.  Calls share the array, so calls whose work overlaps on the GPU
 * (two streams, or two threads) race and give wrong results; serialise them.
 * The cached address does not survive cudaDeviceReset (the reset unloads the
 * array): after a reset, do not call this entry point again in the process.
 * Edge indices are checked on the device, not the host: an edge with an index
 * out of range or with i == j (a self-loop, which the instance format does not
 * allow) is skipped and both outputs become NaN.  The per-node sums of S^T y
 * use FP64 atomic additions, so the lower bound is not bitwise reproducible:
 * its last bits can differ from call to call (the upper bound's do not).
 * Returns 0, PRAQ_ERROR_ARGUMENT for a null pointer, PRAQ_ERROR_INSTANCE for
 * n or m out of range, PRAQ_ERROR_CUDA if a launch failed or if a CUDA error
 * was already pending on the calling thread (it is left pending, and nothing
 * is launched). */
REFORM_API int reform_praq_bounds_noalloc(int64_t n, int64_t m, const double* diag,
                                          const int64_t* rows, const int64_t* cols,
                                          const double* vals, const double* x,
                                          const double* y, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* REFORM_B200_PRAQ_H */
