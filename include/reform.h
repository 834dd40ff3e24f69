/* reform.h -- batched and serving forms of the PRAQ / PRIA solvers.
 *
 * No counterpart in the reference: it solves one instance per call
 * (praq_solve) or fans independent solves out over host threads
 * (pria_solve_batch_*, jrp/pria-cuda/src/pria.cu:15-44).  Here many instances
 * of uneven size -- QUBO and JRP mixed -- share one engine: every kernel
 * launch covers all active instances through device-resident work tables
 * (persistent CTAs and, for the JRP y/z half-step, persistent clusters), each
 * instance keeps its own restart and termination state on the device, one
 * op_steps block of all instances replays as one captured CUDA graph, and
 * finished instances retire between replays by leaving the work tables (no
 * re-capture).  Instances join between blocks, so a serving loop can admit
 * requests while others are running.
 *
 * Every instance computes exactly what its solo solve computes (same kernels,
 * same per-instance layout and order of sums), so results are bitwise those of
 * reform_praq_* / reform_pria_* with the same precision.
 *
 * Precision: iterates in FP32 (use_float32 = 1) or FP64; reductions, restart
 * logic and bounds always FP64.  All instances of a batch share op_steps
 * (the first instance's; default 16); tolerance and max_iter are per instance.
 */
#ifndef REFORM_B200_REFORM_H
#define REFORM_B200_REFORM_H

#include <stdint.h>

#include "praq.h"
#include "pria.h"

#ifndef REFORM_API
#define REFORM_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct reform_batch reform_batch;

/* Tunable launch shapes (reform_batch_autotune picks them; zero = default). */
typedef struct {
    int reserved0;                 /* unused, 0 */
    int grid_multiplier;           /* persistent CTAs per SM for the step kernels: 2..16 */
    int reserved[6];
} reform_shapes;

/* An empty engine on `stream` (cudaStream_t; NULL: a private one). */
REFORM_API int reform_batch_create(int use_float32, void* stream, reform_batch** out);

/* Add an instance: validated and laid out on the device now; it joins the
 * block schedule at reform_batch_start.  Returns its id (>= 0) or a negative
 * error (PRAQ_ERROR_* for QUBO, -(CUDA error) for JRP). */
REFORM_API int reform_batch_add_qubo(reform_batch* b, const PraqInstance* instance,
                                     const PraqParameters* parameters);
REFORM_API int reform_batch_add_jrp(reform_batch* b, int64_t n, int64_t t, const double* order_costs,
                                    double joint_cost, const double* holding_costs,
                                    const pria_params* params);

/* A JRP whose holding costs are demand-driven, H_ist = rate_i d_it (t - s)
 * for s <= t (rate [n], demand [n][t]): the same LP as reform_batch_add_jrp
 * with that dense H, given in N + N T numbers instead of N T^2; the packed
 * costs are built on the device. */
REFORM_API int reform_batch_add_jrp_demand(reform_batch* b, int64_t n, int64_t t, const double* order_costs,
                                           double joint_cost, const double* rate, const double* demand,
                                           const pria_params* params);

/* Cold-start every instance added since the last call (the first vanilla step
 * and the check before the loop) and put it in the work tables. */
REFORM_API int reform_batch_start(reform_batch* b);

/* Run blocks until every instance has terminated (or `max_blocks` blocks,
 * < 0: no cap), retiring instances between replays.  Returns 0 or an error. */
REFORM_API int reform_batch_run(reform_batch* b, int64_t max_blocks);

/* Serving: enqueue one block (a graph replay) without waiting ... */
REFORM_API int reform_batch_launch(reform_batch* b);
/* ... and wait for the oldest enqueued block, retire what it finished, and
 * write up to `max` newly finished ids to `ids` (*count of them).  Returns
 * the number of instances still running, or a negative error. */
REFORM_API int reform_batch_sync(reform_batch* b, int* ids, int max, int* count);

/* Number of blocks enqueued and not yet synced. */
REFORM_API int reform_batch_inflight(const reform_batch* b);

/* Status of instance `id`: done (1 once terminated), iterations, bounds. */
REFORM_API int reform_batch_status(reform_batch* b, int id, int* done, int64_t* iterations,
                                   double* lower, double* upper);

/* Results (any output may be NULL): QUBO primal [n]; JRP dense [n][t][t]. */
REFORM_API int reform_batch_result_qubo(reform_batch* b, int id, double* x, PraqResult* result);
REFORM_API int reform_batch_result_jrp(reform_batch* b, int id, double* x, double* y, double* z,
                                       pria_result_info* info);

/* Free an instance's device memory.  A running instance first leaves the
 * schedule (after the blocks in flight have finished). */
REFORM_API int reform_batch_remove(reform_batch* b, int id);

/* QUBO warm start of an instance added and not yet started (as
 * reform_praq_set_warm: x [n], dual pairs y2 [2m], instance units, projected). */
REFORM_API int reform_batch_set_warm_qubo(reform_batch* b, int id, const double* x, const double* y2);

/* The point of a started QUBO instance's last check (x [n], dual pairs y2
 * [2m], instance units; either may be NULL), running or done: what a warm
 * start elsewhere continues from. */
REFORM_API int reform_batch_point_qubo(reform_batch* b, int id, double* x, double* y2);

/* Device bytes held by the instances of the batch (their layouts and iterates). */
REFORM_API int64_t reform_batch_device_bytes(const reform_batch* b);

/* Launch shapes: set explicitly, or let the autotuner time each candidate on
 * the batch's own instances (one block each, state restarted afterwards) and
 * keep the fastest; `out` receives the choice. */
REFORM_API int reform_batch_set_shapes(reform_batch* b, const reform_shapes* shapes);
REFORM_API int reform_batch_autotune(reform_batch* b, reform_shapes* out);

/* Cold-start every instance that is still held (done or not) again: the
 * instances stay laid out on the device, their iterates start over. */
REFORM_API int reform_batch_restart(reform_batch* b);

/* Kernel launches issued by the engine since creation (graph nodes counted). */
REFORM_API int64_t reform_batch_launches(const reform_batch* b);

REFORM_API void reform_batch_destroy(reform_batch* b);

/* ---- the request server ------------------------------------------------- */

/* A continuous-batching server over the engine above, with its own host
 * thread (no counterpart in the reference; its in-library worker pattern is
 * that of pria_solve_batch_*, jrp/pria-cuda/src/pria.cu:15-44).  Requests are
 * submitted from any thread; the server admits them in arrival order while
 * their estimated device bytes fit the budget (the first one always does),
 * lays them out and starts them between block replays, keeps
 * `blocks_in_flight` blocks queued, and marks converged requests finished
 * after each block.  A finished request keeps its iterates on the device
 * until it is retired; retiring returns its bytes to the budget.  With FP32
 * iterates a QUBO whose gap has not halved over `stall_iterations`
 * iterations continues in an FP64 engine from its last check (its result
 * counts both phases' iterations).  All requests share the options'
 * tolerance and max_iter.  Thread-safe, except that no call may overlap
 * reform_server_destroy. */
typedef struct reform_server reform_server;

typedef struct {
    int64_t budget_bytes;    /* device bytes admitted requests may hold (default 150e9) */
    double tolerance;        /* relative gap (default 1e-4) */
    int64_t max_iter;        /* per request (default 200000; < 0: none) */
    int use_float32;         /* 1 (default): FP32 iterates, FP64 reductions; 0: FP64 */
    int blocks_in_flight;    /* op_steps blocks queued on the GPU (default 2, at most 4) */
    int admit_every;         /* while requests run, admission and retirement at most every
                                this many blocks (default 4; 1 measured the same) */
    int stall_iterations;    /* FP32 QUBO plateau window (default 384; <= 0: never escalate) */
} reform_server_options;

/* A request's state.  Times in seconds since the server was created. */
typedef struct {
    int state;               /* 0 waiting, 1 running, 2 finished, 3 failed */
    int error;               /* a failed request's error (as reform_batch_add_*) */
    int kind;                /* 0 QUBO, 1 JRP */
    int escalated;           /* 1: running or finished in the FP64 engine */
    int64_t iterations;      /* at finish */
    double lower, upper;     /* bracket at finish (instance units) */
    double arrival, admitted, finished;   /* -1 until it happens */
    int64_t device_bytes;    /* its share of the budget */
} reform_server_request;

typedef struct {
    int64_t waiting, running, completed;
    int64_t reserved_bytes, high_water_bytes;   /* budget in use now / at most */
    int64_t device_bytes;                       /* held by the engines now */
    int error;                                  /* nonzero: the loop stopped on this error */
} reform_server_counts;

REFORM_API reform_server_options reform_server_default_options(void);
/* `options` may be NULL (the defaults); fields <= 0 take the defaults. */
REFORM_API int reform_server_create(const reform_server_options* options, reform_server** out);

/* Queue a request; its arrays are copied before the call returns.  Returns
 * the request id (>= 0) or a negative error. */
REFORM_API int64_t reform_server_submit_qubo(reform_server* s, const PraqInstance* instance);
REFORM_API int64_t reform_server_submit_jrp(reform_server* s, int64_t n, int64_t t, const double* order_costs,
                                            double joint_cost, const double* holding_costs);
REFORM_API int64_t reform_server_submit_jrp_demand(reform_server* s, int64_t n, int64_t t,
                                                   const double* order_costs, double joint_cost,
                                                   const double* rate, const double* demand);

/* Ids of requests that finished (or failed) since the last poll: up to `max`
 * into `ids`, their number into *count; each id is reported once.  Waits up to
 * `wait_seconds` for one when there is none.  Returns 0, or the loop's error. */
REFORM_API int reform_server_poll(reform_server* s, int64_t* ids, int max, int* count, double wait_seconds);

REFORM_API int reform_server_status(reform_server* s, int64_t id, reform_server_request* out);

/* Results of a finished request (any output may be NULL), as
 * reform_batch_result_qubo / _jrp. */
REFORM_API int reform_server_result_qubo(reform_server* s, int64_t id, double* x, PraqResult* result);
REFORM_API int reform_server_result_jrp(reform_server* s, int64_t id, double* x, double* y, double* z,
                                        pria_result_info* info);

/* Drop a request: a queued one at once; otherwise its device memory and its
 * share of the budget are released at the loop's next admission turn.  A
 * running request is cancelled. */
REFORM_API int reform_server_retire(reform_server* s, int64_t id);

REFORM_API int reform_server_stats(reform_server* s, reform_server_counts* out);

/* Stops the loop (requests still running are abandoned) and frees everything. */
REFORM_API void reform_server_destroy(reform_server* s);

#ifdef __cplusplus
}
#endif
#endif /* REFORM_B200_REFORM_H */
