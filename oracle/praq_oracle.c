/* praq_oracle.c -- CPU restatement of PRAQ (restarted reflected Halpern PDHG on
 * the QUBO roof-dual LP), FP64, on the SPARSE half-edge set.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA path is checked
 * against and the CPU baseline bench.py times; nothing in the product links or
 * calls it.
 *
 * What it follows (paths inside the MIT-Lu-Lab/reformulation project):
 *   qubo/praq-jax/praq/solver.py:259-273      _raw_step (primal then dual half)
 *   qubo/praq-jax/praq/solver.py:276-292      _reflect_step Halpern combination
 *   qubo/praq-jax/praq/solver.py:320-369      upper/lower bounds, relative gap
 *   qubo/praq-jax/praq/solver.py:372-381      termination (NaN gap keeps going)
 *   qubo/praq-jax/praq/solver.py:397-469      _halpern_step restart + omega logic
 *   qubo/praq-jax/praq/solver.py:483-561      start: projected start, one raw step
 *   qubo/praq-jax/praq/solver.py:199-225      check_interval (Box-Cox rule)
 *   qubo/praq-jax/praq/projection.py:5-42     box clip and the per-edge dual projection
 *   qubo/praq-jax/praq/halpern_operator.py:7-35  canonical norm, + cross term
 *   qubo/praq-jax/praq/half_edge.py:42-99     degree floor, shift, centroid start
 *   qubo/praq-cuda/src/solver.cuh:31-41,517-569  sparse degree (true incident
 *                                             count, floored at 1), signed 2 W_ij
 *   qubo/praq-cuda/src/solver.cuh:716-783     host loop: the restart takes one
 *                                             uncounted vanilla step; the point
 *                                             returned is the one the gap was
 *                                             measured at; bounds at the
 *                                             original scale
 *   qubo/praq-cuda/src/praq.cu:35-79          argument and instance validation
 *
 * The warm phase of solve_qubo_problem_warm_start runs op_steps * warm_steps
 * = 0 vanilla steps with the defaults, and leaves omega unchanged, so it is a
 * no-op and is not restated (praq-cuda omits it for the same reason).
 *
 * Threads: with threads > 1 the node and edge loops run under OpenMP.  Every
 * per-element update is independent; the sums are accumulated per thread over
 * a static partition and added in thread order, so a run is deterministic for
 * a given thread count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_EXPORT __attribute__((visibility("default")))

/* Parameter block, in the field order of the reference's PraqParameters
 * (qubo/praq-cuda/include/praq/praq.h:29-60). */
typedef struct {
    double tolerance;
    int64_t max_iter;
    int use_float32;
    double omega;
    double beta_sufficient;
    double beta_necessary;
    double beta_artificial;
    double theta_initial;
    double theta_target;
    double theta_decay;
    int64_t op_steps;
    double interval_offset;
    double interval_scale;
    double interval_power;
} OracleParams;

static const double kEta = 0.999;   /* 0.999 / ||A||, ||A|| = 1 for PRAQ */

ORACLE_EXPORT int64_t oracle_check_interval(int64_t n, double offset, double scale,
                                            double power) {
    double u = log((double)n / 50000.0);
    double b = power == 0.0 ? u : expm1(power * u) / power;
    double v = floor(offset + scale * b + 0.5);
    if (!(v >= 2.0)) return 2;
    if (v > 1e9) return 1000000000;
    return (int64_t)v;
}

typedef struct {
    int64_t n, m;
    double scale;
    int64_t *ptr, *half;       /* CSR incidence: half-edges 2e + slot */
    int64_t *e0, *e1;
    double *w, *diag, *deg;    /* w signed, 2 W_ij / scale */
    int threads;
} Graph;

typedef struct {
    double *x, *sx, *x0;       /* point stepped from, the step, the anchor */
    double *y, *sy, *y0;       /* pairs, [2m] */
    double *st;                /* scatter scratch [n] */
    double *r;                 /* reflected primal [n] */
} Iterates;

static double clamp(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

static int nthreads(const Graph* g) { return g->threads > 0 ? g->threads : 1; }

/* (S^T y)_i: the sum of a node's incident half-edge duals, in CSR order. */
static void scatter(const Graph* g, const double* y, double* out) {
    int64_t n = g->n;
#pragma omp parallel for schedule(static) num_threads(nthreads(g))
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int64_t k = g->ptr[i]; k < g->ptr[i + 1]; ++k) s += y[g->half[k]];
        out[i] = s;
    }
}

/* One PDHG step (_raw_step): (x1, y1) -> (x2, y2). */
static void raw_step(const Graph* g, Iterates* it, const double* x1, const double* y1,
                     double* x2, double* y2, double omega) {
    int64_t n = g->n, m = g->m;
    double primal_step = kEta / omega, dual_step = kEta * omega;
    scatter(g, y1, it->st);
#pragma omp parallel for schedule(static) num_threads(nthreads(g))
    for (int64_t i = 0; i < n; ++i) {
        double gradient = g->diag[i] - it->st[i];
        double v = clamp(x1[i] - primal_step * (gradient / g->deg[i]), 0.0, 1.0);
        x2[i] = v;
        it->r[i] = 2.0 * v - x1[i];
    }
#pragma omp parallel for schedule(static) num_threads(nthreads(g))
    for (int64_t e = 0; e < m; ++e) {
        double sw = g->w[e], w = fabs(sw);
        int positive = sw > 0.0;
        double a = y1[2 * e] + dual_step * ((positive ? 1.0 : 0.0) - it->r[g->e0[e]]);
        double b = y1[2 * e + 1] + dual_step * (0.0 - it->r[g->e1[e]]);
        if (positive) {
            double mu = clamp(0.5 * (a + b), -w, 0.0);
            y2[2 * e] = mu;
            y2[2 * e + 1] = mu;
        } else {
            double first = clamp(a + 0.5 * (w - a - b), 0.0, w);
            y2[2 * e] = first;
            y2[2 * e + 1] = w - first;
        }
    }
}

/* The check sums: canonical-norm pieces of (x - sx, y - sy), drifts from the
 * anchor, and both bounds at (bx, by), in scaled units. */
typedef struct {
    double primal_norm, dual_norm, cross, primal_drift, dual_drift;
    double upper, lower;
} Sums;

static Sums check_sums(const Graph* g, Iterates* it, const double* bx, const double* by) {
    int64_t n = g->n, m = g->m;
    int T = nthreads(g);
    double* part = (double*)calloc((size_t)T * 8, sizeof(double));
    scatter(g, by, it->st);
#pragma omp parallel num_threads(T)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
#pragma omp for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            double dx = it->x[i] - it->sx[i], dr = it->x[i] - it->x0[i];
            a0 += g->deg[i] * dx * dx;
            a3 += g->deg[i] * dr * dr;
            a5 += g->diag[i] * bx[i];
            double rc = g->diag[i] - it->st[i];
            a6 += rc < 0.0 ? rc : 0.0;
        }
        double b1 = 0, b2 = 0, b4 = 0, b5 = 0, b6 = 0;
#pragma omp for schedule(static)
        for (int64_t e = 0; e < m; ++e) {
            int64_t i = g->e0[e], j = g->e1[e];
            double sw = g->w[e], w = fabs(sw);
            double dya = it->y[2 * e] - it->sy[2 * e], dyb = it->y[2 * e + 1] - it->sy[2 * e + 1];
            b1 += dya * dya + dyb * dyb;
            b2 += (it->x[i] - it->sx[i]) * dya + (it->x[j] - it->sx[j]) * dyb;
            double ra = it->y[2 * e] - it->y0[2 * e], rb = it->y[2 * e + 1] - it->y0[2 * e + 1];
            b4 += ra * ra + rb * rb;
            if (sw > 0.0) {
                b5 += w * fmax(bx[i] + bx[j] - 1.0, 0.0);
                b6 += by[2 * e];
            } else {
                b5 += -w * fmin(bx[i], bx[j]);
            }
        }
        double* p = part + (size_t)tid * 8;
        p[0] = a0; p[1] = b1; p[2] = b2; p[3] = a3; p[4] = b4;
        p[5] = a5 + b5; p[6] = a6 + b6;
        (void)a1; (void)a2; (void)a4;
    }
    Sums s = {0, 0, 0, 0, 0, 0, 0};
    for (int t = 0; t < T; ++t) {
        double* p = part + (size_t)t * 8;
        s.primal_norm += p[0];
        s.dual_norm += p[1];
        s.cross += p[2];
        s.primal_drift += p[3];
        s.dual_drift += p[4];
        s.upper += p[5];
        s.lower += p[6];
    }
    free(part);
    return s;
}

static double canonical_norm(const Sums* s, double omega) {
    double v = (omega / kEta) * s->primal_norm + (1.0 / (kEta * omega)) * s->dual_norm
             + 2.0 * s->cross;
    return sqrt(v > 0.0 ? v : 0.0);
}

static int should_stop(double gap, int64_t iteration, int64_t max_iter, double tol) {
    int within = iteration < max_iter || max_iter < 0;
    int outside = !(gap <= tol);
    return !(within && outside);
}

static void copy(double* dst, const double* src, int64_t count) {
    memcpy(dst, src, sizeof(double) * (size_t)count);
}

/* Solve.  out[0..4) = lower, upper, iterations, status.  Returns the status:
 * 0 converged, 1 iteration limit, -1 argument, -2 instance. */
ORACLE_EXPORT int oracle_praq_solve(int64_t n, int64_t m, const double* diag,
                                    const int64_t* rows, const int64_t* cols,
                                    const double* vals, const OracleParams* params,
                                    int threads, double* x_out, double* y_out, double* out) {
    out[0] = NAN; out[1] = NAN; out[2] = 0; out[3] = -1;
    if (!params || !x_out) return -1;
    OracleParams p = *params;
    if (!(p.tolerance >= 0.0) || !(p.omega > 0.0) || !(p.beta_sufficient > 0.0)
        || !(p.beta_necessary > 0.0) || !(p.beta_artificial >= 0.0)
        || !isfinite(p.theta_initial) || !isfinite(p.theta_target) || !isfinite(p.theta_decay)
        || !isfinite(p.interval_offset) || !isfinite(p.interval_scale)
        || !(p.interval_power >= 0.0)) return -1;
    if (n <= 0 || m < 0 || !diag || (m > 0 && (!rows || !cols || !vals))) { out[3] = -2; return -2; }
    for (int64_t e = 0; e < m; ++e) {
        if (rows[e] < 0 || rows[e] >= n || cols[e] < 0 || cols[e] >= n || rows[e] == cols[e]) {
            out[3] = -2;
            return -2;
        }
    }
    if (p.max_iter <= 0) p.max_iter = -1;
    if (p.op_steps <= 0) p.op_steps = oracle_check_interval(n, p.interval_offset,
                                                          p.interval_scale, p.interval_power);
    if (p.op_steps < 2) p.op_steps = 2;

    Graph g;
    g.n = n; g.m = m; g.threads = threads;
    g.e0 = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m + 1));
    g.e1 = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m + 1));
    g.w = (double*)malloc(sizeof(double) * (size_t)(m + 1));
    g.diag = (double*)malloc(sizeof(double) * (size_t)n);
    g.deg = (double*)malloc(sizeof(double) * (size_t)n);
    g.ptr = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    g.half = (int64_t*)malloc(sizeof(int64_t) * (size_t)(2 * m + 1));
    double squares = 0.0;
    for (int64_t i = 0; i < n; ++i) squares += diag[i] * diag[i];
    for (int64_t e = 0; e < m; ++e) {
        g.e0[e] = rows[e];
        g.e1[e] = cols[e];
        g.w[e] = 2.0 * vals[e];
        squares += g.w[e] * g.w[e];
    }
    g.scale = squares > 0.0 ? sqrt(squares) : 1.0;
    for (int64_t i = 0; i < n; ++i) g.diag[i] = diag[i] / g.scale;
    for (int64_t e = 0; e < m; ++e) g.w[e] /= g.scale;
    for (int64_t e = 0; e < m; ++e) { ++g.ptr[g.e0[e] + 1]; ++g.ptr[g.e1[e] + 1]; }
    for (int64_t i = 0; i < n; ++i) g.ptr[i + 1] += g.ptr[i];
    {
        int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
        memcpy(fill, g.ptr, sizeof(int64_t) * (size_t)n);
        for (int64_t e = 0; e < m; ++e) {
            g.half[fill[g.e0[e]]++] = 2 * e;
            g.half[fill[g.e1[e]]++] = 2 * e + 1;
        }
        free(fill);
    }
    for (int64_t i = 0; i < n; ++i) {
        int64_t d = g.ptr[i + 1] - g.ptr[i];
        g.deg[i] = d > 0 ? (double)d : 1.0;
    }

    Iterates it;
    it.x = (double*)malloc(sizeof(double) * (size_t)n);
    it.sx = (double*)malloc(sizeof(double) * (size_t)n);
    it.x0 = (double*)malloc(sizeof(double) * (size_t)n);
    it.st = (double*)malloc(sizeof(double) * (size_t)n);
    it.r = (double*)malloc(sizeof(double) * (size_t)n);
    it.y = (double*)malloc(sizeof(double) * (size_t)(2 * m + 2));
    it.sy = (double*)malloc(sizeof(double) * (size_t)(2 * m + 2));
    it.y0 = (double*)malloc(sizeof(double) * (size_t)(2 * m + 2));
    double* tx = (double*)malloc(sizeof(double) * (size_t)n);
    double* ty = (double*)malloc(sizeof(double) * (size_t)(2 * m + 2));

    /* Cold start: the centroid, x = 1/2 and y_e = (-W_ij, -W_ij) (scaled). */
    for (int64_t i = 0; i < n; ++i) it.x0[i] = 0.5;
    for (int64_t e = 0; e < m; ++e) {
        it.y0[2 * e] = -0.5 * g.w[e];
        it.y0[2 * e + 1] = -0.5 * g.w[e];
    }
    double omega = p.omega, theta = p.theta_initial;
    int64_t iteration = 0, restart_iter = 0;
    copy(it.x, it.x0, n);
    copy(it.y, it.y0, 2 * m);
    raw_step(&g, &it, it.x, it.y, it.sx, it.sy, omega);

    Sums s = check_sums(&g, &it, it.x, it.y);
    double fp_error = canonical_norm(&s, omega);
    double check_error = INFINITY;
    double upper = s.upper * g.scale, lower = s.lower * g.scale;
    double gap = (upper - lower) / (1.0 + fabs(upper) + fabs(lower));
    int terminated = should_stop(gap, iteration, p.max_iter, p.tolerance);

    while (!terminated) {
        for (int64_t k = 0; k < p.op_steps; ++k) {
            double kk = (double)(restart_iter + 1);
            double lw = kk / (kk + 1.0), rw = 1.0 / (kk + 1.0);
#pragma omp parallel for schedule(static) num_threads(nthreads(&g))
            for (int64_t i = 0; i < n; ++i) tx[i] = lw * (2.0 * it.sx[i] - it.x[i]) + rw * it.x0[i];
#pragma omp parallel for schedule(static) num_threads(nthreads(&g))
            for (int64_t h = 0; h < 2 * m; ++h) ty[h] = lw * (2.0 * it.sy[h] - it.y[h]) + rw * it.y0[h];
            copy(it.x, tx, n);
            copy(it.y, ty, 2 * m);
            raw_step(&g, &it, it.x, it.y, it.sx, it.sy, omega);
            ++restart_iter;
            ++iteration;
        }
        s = check_sums(&g, &it, it.sx, it.sy);
        double new_error = canonical_norm(&s, omega);
        upper = s.upper * g.scale;
        lower = s.lower * g.scale;
        gap = (upper - lower) / (1.0 + fabs(upper) + fabs(lower));
        terminated = should_stop(gap, iteration, p.max_iter, p.tolerance);

        int sufficient = new_error <= p.beta_sufficient * fp_error;
        int necessary = new_error <= p.beta_necessary * fp_error && new_error > check_error;
        int artificial = (double)restart_iter >= p.beta_artificial * (double)iteration;
        int restart = sufficient || necessary || artificial;
        if (restart) {
            double pn = sqrt(s.primal_drift), dn = sqrt(s.dual_drift);
            if (pn > 1e-16 && dn > 1e-16) {
                omega = exp(theta * (log(dn) - log(pn)) + (1.0 - theta) * log(omega));
                theta = p.theta_target + p.theta_decay * (theta - p.theta_target);
            }
        }
        if (terminated) {
            copy(it.x, it.sx, n);
            copy(it.y, it.sy, 2 * m);
            break;
        }
        if (restart) {
            copy(it.x, it.sx, n);
            copy(it.y, it.sy, 2 * m);
            raw_step(&g, &it, it.x, it.y, it.sx, it.sy, omega);
            copy(it.x0, it.x, n);
            copy(it.y0, it.y, 2 * m);
            Sums r = check_sums(&g, &it, it.sx, it.sy);
            fp_error = canonical_norm(&r, omega);
            check_error = INFINITY;
            restart_iter = 0;
        } else {
            check_error = new_error;
        }
    }

    for (int64_t i = 0; i < n; ++i) x_out[i] = it.x[i];
    if (y_out) for (int64_t h = 0; h < 2 * m; ++h) y_out[h] = it.y[h] * g.scale;
    int status = gap <= p.tolerance ? 0 : 1;
    out[0] = lower;
    out[1] = upper;
    out[2] = (double)iteration;
    out[3] = status;

    free(g.e0); free(g.e1); free(g.w); free(g.diag); free(g.deg); free(g.ptr); free(g.half);
    free(it.x); free(it.sx); free(it.x0); free(it.st); free(it.r);
    free(it.y); free(it.sy); free(it.y0); free(tx); free(ty);
    return status;
}

/* F(x) of the relaxation at x, in the instance's own units (the upper bound
 * of qubo/praq-jax/praq/solver.py:320-328, unscaled), for certificate checks. */
ORACLE_EXPORT double oracle_praq_relaxation_value(int64_t n, int64_t m, const double* diag,
                                                  const int64_t* rows, const int64_t* cols,
                                                  const double* vals, const double* x) {
    double v = 0.0;
    for (int64_t i = 0; i < n; ++i) v += diag[i] * x[i];
    for (int64_t e = 0; e < m; ++e) {
        double xi = x[rows[e]], xj = x[cols[e]], w = 2.0 * vals[e];
        v += w > 0.0 ? w * fmax(xi + xj - 1.0, 0.0) : w * fmin(xi, xj);
    }
    return v;
}
