/* pria.h -- C ABI of the B200 PRIA solver (the joint replenishment LP by
 * restarted, reflected Halpern PDHG on upper-triangular simplices).
 *
 *   minimize    sum_s K0 z_s + sum_{i,s} K_i y_is + sum_{i,t} sum_{s<=t} H_ist x_ist
 *   subject to  sum_{s<=t} x_ist = 1,  x_ist <= y_is,  x_ist <= z_s,  x, y, z >= 0
 *
 * The first block is a drop-in for the reference's libpria.so: the same entry
 * points, struct layouts and argument meaning.
 *
 *   pria_params / pria_result_info   replace jrp/pria-cuda/include/pria/pria.h:34-59
 *   pria_params_auto                 replaces jrp/pria-cuda/include/pria/pria.h:52
 *                                    (defaults of Parameters.with_auto_step,
 *                                    jrp/pria-jax/pria/solver.py:150-188)
 *   pria_solve_f64 / pria_solve_f32  replace jrp/pria-cuda/include/pria/pria.h:75-85
 *   pria_solve_batch_f64 / _f32      replace jrp/pria-cuda/include/pria/pria.h:95-105
 *   pria_objective_f64               replaces jrp/pria-cuda/include/pria/pria.h:110-112
 *
 * Conventions (as the reference's): H is dense row-major [n][t][t], only s <= t
 * read; outputs x, y, z are dense [n][t][t], upper triangular; the returned y
 * and z are normalised by K_i and K0 (rows of y sum to 1 over t >= s, each z
 * group {i, t >= s} sums to 1), so a returned triple warm-starts as the fixed
 * point it is.  An odd t is padded by one period of zero holding cost.
 *
 * pria_result_info: primal_objective is the objective at the returned
 * (unpadded) x, an upper bound; dual_objective is the padded dual bound the
 * solver converged against, a lower bound; relative_gap is formed from those
 * two.  (jrp/pria-jax/pria/solver.py:613-631 explains the split.)
 *
 * Returns 0 or a nonzero CUDA error code (cudaErrorInvalidValue for n < 1,
 * t < 1, a null order_costs/holding_costs/params, a padded period count above
 * 1024, or an instance too large for int64 indexing).  pria_solve_f32 iterates
 * in FP32 and keeps every reduction, the restart logic and the bounds in FP64.
 * Thread-safe: each call uses its own stream and never the legacy stream.
 */
#ifndef REFORM_B200_PRIA_H
#define REFORM_B200_PRIA_H

#include <stdint.h>

#include "reform_trace.h"

#ifndef REFORM_API
#define REFORM_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pria_params {
    double omega;            /* initial primal weight */
    double eta;              /* step size */
    double beta_sufficient;  /* sufficient-decay restart threshold */
    double beta_artificial;  /* artificial restart threshold */
    double beta_necessary;   /* necessary restart threshold */
    double theta_initial;    /* initial primal-weight smoothing exponent */
    double theta_target;     /* exponent theta decays toward */
    double theta_decay;      /* fraction of remaining theta gap kept per update */
    double tolerance;        /* relative optimality tolerance */
    int64_t max_iter;        /* maximum operator steps, -1 for unlimited */
    int use_halpern;         /* nonzero: restarted Halpern; zero: vanilla PDHG */
    int warm_steps;          /* vanilla op_steps blocks to run before Halpern */
    int op_steps;            /* operator steps between convergence checks */
    int verbose;             /* nonzero: per-check progress on stderr */
} pria_params;

typedef struct pria_result_info {
    int64_t iterations;      /* operator steps performed */
    double primal_objective; /* objective at the returned x (upper bound) */
    double dual_objective;   /* dual bound (lower bound) */
    double relative_gap;     /* (primal - dual) / (1 + |primal| + |dual|) */
} pria_result_info;

REFORM_API pria_params pria_params_auto(int64_t max_iter, double tolerance);

REFORM_API int pria_solve_f64(int64_t n, int64_t t, const double* order_costs, double joint_cost,
                              const double* holding_costs, const pria_params* params,
                              const double* warm_x, const double* warm_y, const double* warm_z,
                              double* x, double* y, double* z, pria_result_info* info);

REFORM_API int pria_solve_f32(int64_t n, int64_t t, const float* order_costs, float joint_cost,
                              const float* holding_costs, const pria_params* params,
                              const float* warm_x, const float* warm_y, const float* warm_z,
                              float* x, float* y, float* z, pria_result_info* info);

REFORM_API int pria_solve_batch_f64(int64_t count, int64_t n, int64_t t, const double* order_costs,
                                    const double* joint_costs, const double* holding_costs,
                                    const pria_params* params, double* x, double* y, double* z,
                                    pria_result_info* infos);

REFORM_API int pria_solve_batch_f32(int64_t count, int64_t n, int64_t t, const float* order_costs,
                                    const float* joint_costs, const float* holding_costs,
                                    const pria_params* params, float* x, float* y, float* z,
                                    pria_result_info* infos);

REFORM_API double pria_objective_f64(int64_t n, int64_t t, const double* order_costs,
                                     double joint_cost, const double* holding_costs,
                                     const double* x);

/* ---- device-resident solves (no reference counterpart) ------------------- */

typedef struct reform_pria_solver reform_pria_solver;

/* Lay an instance out on the device (FP64 input; `use_float32` selects FP32
 * iterates with FP64 reductions) on `stream` (a cudaStream_t; NULL: a private
 * non-blocking stream).  Returns 0 or a CUDA error code. */
REFORM_API int reform_pria_create(int64_t n, int64_t t, const double* order_costs,
                                  double joint_cost, const double* holding_costs,
                                  const pria_params* params, int use_float32, void* stream,
                                  reform_pria_solver** out);

/* One full solve from the cold start (or from the warm start last given with
 * reform_pria_set_warm).  Blocks the host until done.  Returns 0, a CUDA
 * error code, or REFORM_PRIA_STATUS_TIME_LIMIT (below). */
REFORM_API int reform_pria_run(reform_pria_solver* solver);

/* A wall-clock budget for each run, in seconds (< 0: none, the default); no
 * counterpart in the reference's library, whose harness kills the solver
 * process past the limit (jrp/harness/backends/pria_cuda.py:114-145).  The
 * host checks it each time a convergence check's result arrives; when it has
 * run out, the run stops there (the block already in flight finishes) and
 * returns REFORM_PRIA_STATUS_TIME_LIMIT, and reform_pria_result gives the point
 * and the bracket of the last completed check -- a valid bracket, since every
 * iterate is feasible.  A run that converges in the same block returns 0. */
#define REFORM_PRIA_STATUS_TIME_LIMIT (-1)
/* Only from a library built with RB200_DEBUG_BOUNDS (python -m
 * reformulation_b200.build --debug-bounds): an index out of range was caught
 * and its access skipped; the result is not valid. */
#define REFORM_PRIA_STATUS_BOUNDS (-2)
REFORM_API int reform_pria_set_time_limit(reform_pria_solver* solver, double seconds);

/* Warm start for the next runs: dense [n][t][t] FP64 arrays in the output
 * convention (duals normalised); NULL pointers clear it. */
REFORM_API int reform_pria_set_warm(reform_pria_solver* solver, const double* warm_x,
                                    const double* warm_y, const double* warm_z);

/* The last run's solution (any pointer may be NULL), dense [n][t][t] FP64. */
REFORM_API int reform_pria_result(reform_pria_solver* solver, double* x, double* y, double* z,
                                  pria_result_info* info);

/* A measurement run: every kernel between a pair of CUDA events on the
 * solver's stream; ms[9]/count[9] receive each kind's total device time and
 * launches: x step, y/z step, x step with check sums, y/z step with check
 * sums, upper bound, lower bound, check, restart (x, y/z, check together),
 * and a whole check block of the persistent kernel (below). */
REFORM_API int reform_pria_run_profiled(reform_pria_solver* solver, double* ms, int64_t* count);

/* Small instances (the reference's megakernel, jrp/pria-cuda/src/solver.cuh:
 * 145-312, PRIA_MEGA): a check block runs as ONE cooperative launch whose
 * phases (x; y and z; bounds; check; restart step) are separated by grid
 * barriers, in place of the captured graph of one kernel per phase.  `mode`
 * -1: automatic (the default; on for at most 16,384 packed entries, the sizes
 * where it measured at least as fast as the graph), 0: off, 1: on whenever
 * the instance allows it (every z period block within one CTA's shared
 * memory).  The environment variable REFORM_PRIA_MEGA=0|1 sets the mode at
 * creation.  *active (may be NULL) receives 1 when later runs take the
 * persistent kernel.  Results equal the graph's bit for bit in FP64 (the same
 * tile functions and sums); FP32 z sums are taken over 256-thread CTAs
 * instead of 512, so low bits may differ.  Every barrier wait is bounded (1 s
 * of device time): one that runs out ends the launch, and the run returns
 * cudaErrorLaunchTimeout (702) with the context still usable. */
REFORM_API int reform_pria_set_megakernel(reform_pria_solver* solver, int mode, int* active);

/* The convergence trace (include/reform_trace.h): later runs write one record
 * per convergence check -- the start check, every op_steps block, and in the
 * vanilla phase its blocks and its end -- into a device ring of `capacity`
 * records (0: no trace, the default), from the start of each run.  Setting it
 * drops the solver's captured block (the next run captures a new one).
 * Returns 0 or a CUDA error code. */
REFORM_API int reform_pria_set_trace(reform_pria_solver* solver, int capacity);

/* The last run's trace, oldest first: the most recent min(written, ring
 * capacity, `capacity`) records into `out`; *total (may be NULL) receives the
 * number the run wrote. */
REFORM_API int reform_pria_trace(reform_pria_solver* solver, reform_trace_record* out, int capacity,
                                 int64_t* total);

REFORM_API int64_t reform_pria_launches(const reform_pria_solver* solver);

REFORM_API void reform_pria_destroy(reform_pria_solver* solver);

#ifdef __cplusplus
}
#endif
#endif /* REFORM_B200_PRIA_H */
