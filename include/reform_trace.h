/* reform_trace.h -- the convergence trace record shared by the PRAQ and PRIA
 * solvers (reform_praq_set_trace / reform_pria_set_trace).
 *
 * No counterpart in the reference's C libraries, whose `verbose` flag prints
 * one line per check to stderr; the JAX solvers queue the same facts through
 * jax.debug.callback (jrp/pria-jax/pria/convergence_log.py:25-97).  Here the
 * device writes one record per convergence check into a ring the caller sizes,
 * with no host involvement while the solve runs; the caller reads it after.
 */
#ifndef REFORM_B200_TRACE_H
#define REFORM_B200_TRACE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* `restart`: what the check decided --
 *   -1  the check before the first step (the start point)
 *    0  no restart
 *    1  restart on sufficient decay of the fixed-point error
 *    2  restart on necessary decay (the error grew since the last check)
 *    3  artificial restart (the iterations since the last restart reached
 *       beta_artificial of all iterations)
 *    4  a check of the plain-PDHG (vanilla) phase
 *    5  the end of the vanilla phase, where the Halpern method starts
 * `terminated` is 1 on the check that ended the solve (tolerance or iteration
 * limit; a restart decided there is not taken). */
typedef struct reform_trace_record {
    int64_t iteration;   /* operator steps done */
    double gap;          /* relative duality gap at the check */
    double error;        /* fixed-point (canonical-norm) error at the check;
                            NaN at the checks of a vanilla phase */
    double omega;        /* primal weight after the check's update */
    double lower;        /* dual bound, instance units */
    double upper;        /* primal bound, instance units */
    int32_t restart;
    int32_t terminated;
} reform_trace_record;

#ifdef __cplusplus
}
#endif
#endif /* REFORM_B200_TRACE_H */
