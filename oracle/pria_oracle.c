/* pria_oracle.c -- CPU restatement of PRIA (restarted reflected Halpern PDHG on
 * the joint replenishment LP), FP64.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against and a CPU baseline bench.py may time; nothing in the product links or
 * calls it.
 *
 * What it follows (paths inside the MIT-Lu-Lab/reformulation project):
 *   jrp/pria-jax/pria/solver.py:409-425     _raw_step: x' = P_X(x - tau(h + y + z)),
 *                                           r = sigma(2x' - x), y' = P_Y(y + r),
 *                                           z' = P_Z(z + r)
 *   jrp/pria-jax/pria/solver.py:428-447     Halpern combination
 *   jrp/pria-jax/pria/solver.py:347-402     upper (primal) and lower (dual) bounds
 *   jrp/pria-jax/pria/solver.py:473-493     relative gap, termination (NaN keeps going)
 *   jrp/pria-jax/pria/solver.py:514-594     restart tests, omega/theta update
 *   jrp/pria-jax/pria/solver.py:608-724     padding of odd T, scaling, projected
 *                                           start, output normalisation
 *   jrp/pria-jax/pria/projection.py:5-30    sort-based simplex projection
 *                                           (Blondel, Fujino and Ueda); a
 *                                           nonpositive target maps to {0}
 *   jrp/pria-jax/pria/halpern_operator.py:5-19  canonical norm, NEGATIVE cross term
 *   jrp/pria-jax/pria/solver.py:150-188     defaults (omega 0.10835, eta 0.999/sqrt 2)
 *   jrp/pria-cuda/tests/ref_impl.hpp:237-422  the same control flow in C++, used
 *                                           here as a cross-check (see oracle/Makefile)
 *
 * Storage: every variable is kept on the padded upper triangle, item-major and
 * row-major inside an item: entry (i, s, t), s <= t < Tp, sits at
 * i * P + off(s) + (t - s) with off(s) = s Tp - s (s - 1) / 2 and
 * P = Tp (Tp + 1) / 2.
 *
 * Threads: with threads > 1 the per-segment loops run under OpenMP; sums are
 * taken per thread over a static partition and added in thread order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_EXPORT __attribute__((visibility("default")))

/* Field order of the reference's pria_params (jrp/pria-cuda/include/pria/pria.h:34-49). */
typedef struct {
    double omega, eta, beta_sufficient, beta_artificial, beta_necessary;
    double theta_initial, theta_target, theta_decay, tolerance;
    int64_t max_iter;
    int use_halpern, warm_steps, op_steps, verbose;
} OraclePriaParams;

typedef struct {
    int64_t n, t, tp, P;
    int64_t ND;
    double scale, k0;
    double *k, *h;   /* scaled */
    int threads;
} Shape;

static inline int64_t off(const Shape* d, int64_t s) { return s * d->tp - s * (s - 1) / 2; }
static inline int64_t at(const Shape* d, int64_t i, int64_t s, int64_t t) {
    return i * d->P + off(d, s) + (t - s);
}
static int nth(const Shape* d) { return d->threads > 0 ? d->threads : 1; }

static int desc(const void* a, const void* b) {
    double x = *(const double*)a, y = *(const double*)b;
    return x < y ? 1 : (x > y ? -1 : 0);
}

/* Euclidean projection of v[0..len) onto {u >= 0, sum u = target}; a
 * nonpositive target gives the zero vector.  `work` holds len doubles. */
static void simplex(double* v, int64_t len, double target, double* work) {
    if (len <= 0) return;
    if (!(target > 0.0)) {
        for (int64_t k = 0; k < len; ++k) v[k] = 0.0;
        return;
    }
    memcpy(work, v, sizeof(double) * (size_t)len);
    qsort(work, (size_t)len, sizeof(double), desc);
    double running = 0.0, theta = INFINITY;
    int64_t rho = 0;
    double cum_rho = 0.0;
    for (int64_t k = 0; k < len; ++k) {
        running += work[k];
        if (work[k] * (double)(k + 1) > running - target) {
            rho = k + 1;
            cum_rho = running;
        }
    }
    if (rho > 0) theta = (cum_rho - target) / (double)rho;
    for (int64_t k = 0; k < len; ++k) {
        double u = v[k] - theta;
        v[k] = u > 0.0 ? u : 0.0;
    }
}

/* P_X: per (i, t), the column {x_ist : s <= t} onto the unit simplex. */
static void proj_x(const Shape* d, double* x) {
#pragma omp parallel num_threads(nth(d))
    {
        double* seg = (double*)malloc(sizeof(double) * (size_t)d->tp);
        double* work = (double*)malloc(sizeof(double) * (size_t)d->tp);
#pragma omp for schedule(static) collapse(2)
        for (int64_t i = 0; i < d->n; ++i)
            for (int64_t t = 0; t < d->tp; ++t) {
                for (int64_t s = 0; s <= t; ++s) seg[s] = x[at(d, i, s, t)];
                simplex(seg, t + 1, 1.0, work);
                for (int64_t s = 0; s <= t; ++s) x[at(d, i, s, t)] = seg[s];
            }
        free(seg);
        free(work);
    }
}

/* P_Y: per (i, s), the row {y_ist : t >= s} onto the K_i simplex. */
static void proj_y(const Shape* d, double* y) {
#pragma omp parallel num_threads(nth(d))
    {
        double* work = (double*)malloc(sizeof(double) * (size_t)d->tp);
#pragma omp for schedule(static) collapse(2)
        for (int64_t i = 0; i < d->n; ++i)
            for (int64_t s = 0; s < d->tp; ++s)
                simplex(y + at(d, i, s, s), d->tp - s, d->k[i], work);
        free(work);
    }
}

/* P_Z: per s, the group {z_ist : all i, t >= s} onto the K0 simplex. */
static void proj_z(const Shape* d, double* z) {
#pragma omp parallel num_threads(nth(d))
    {
        int64_t cap = d->n * d->tp;
        double* seg = (double*)malloc(sizeof(double) * (size_t)cap);
        double* work = (double*)malloc(sizeof(double) * (size_t)cap);
#pragma omp for schedule(dynamic, 1)
        for (int64_t s = 0; s < d->tp; ++s) {
            int64_t w = d->tp - s, p = 0;
            for (int64_t i = 0; i < d->n; ++i)
                for (int64_t t = s; t < d->tp; ++t) seg[p++] = z[at(d, i, s, t)];
            simplex(seg, d->n * w, d->k0, work);
            p = 0;
            for (int64_t i = 0; i < d->n; ++i)
                for (int64_t t = s; t < d->tp; ++t) z[at(d, i, s, t)] = seg[p++];
        }
        free(seg);
        free(work);
    }
}

typedef struct { double *x, *y, *z; } Trio;

static void trio_alloc(Trio* a, int64_t nd) {
    a->x = (double*)calloc((size_t)nd, sizeof(double));
    a->y = (double*)calloc((size_t)nd, sizeof(double));
    a->z = (double*)calloc((size_t)nd, sizeof(double));
}
static void trio_free(Trio* a) { free(a->x); free(a->y); free(a->z); }
static void trio_copy(Trio* dst, const Trio* src, int64_t nd) {
    memcpy(dst->x, src->x, sizeof(double) * (size_t)nd);
    memcpy(dst->y, src->y, sizeof(double) * (size_t)nd);
    memcpy(dst->z, src->z, sizeof(double) * (size_t)nd);
}

/* One PDHG operator application, in -> out. */
static void raw_step(const Shape* d, double omega, double eta, const Trio* in, Trio* out) {
    double tau = eta / omega, sigma = eta * omega;
    int64_t nd = d->ND;
#pragma omp parallel for schedule(static) num_threads(nth(d))
    for (int64_t g = 0; g < nd; ++g) out->x[g] = in->x[g] - tau * (d->h[g] + in->y[g] + in->z[g]);
    proj_x(d, out->x);
#pragma omp parallel for schedule(static) num_threads(nth(d))
    for (int64_t g = 0; g < nd; ++g) {
        double r = sigma * (2.0 * out->x[g] - in->x[g]);
        out->y[g] = in->y[g] + r;
        out->z[g] = in->z[g] + r;
    }
    proj_y(d, out->y);
    proj_z(d, out->z);
}

/* sum dx^2, sum dy^2 + dz^2, sum dx (dy + dz) over a - b. */
static void diffs(const Shape* d, const Trio* a, const Trio* b, double* s3) {
    int T = nth(d);
    double* part = (double*)calloc((size_t)T * 3, sizeof(double));
#pragma omp parallel num_threads(T)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double a0 = 0, a1 = 0, a2 = 0;
#pragma omp for schedule(static)
        for (int64_t g = 0; g < d->ND; ++g) {
            double dx = a->x[g] - b->x[g], dy = a->y[g] - b->y[g], dz = a->z[g] - b->z[g];
            a0 += dx * dx;
            a1 += dy * dy + dz * dz;
            a2 += dx * (dy + dz);
        }
        part[3 * tid] = a0; part[3 * tid + 1] = a1; part[3 * tid + 2] = a2;
    }
    s3[0] = s3[1] = s3[2] = 0.0;
    for (int t = 0; t < T; ++t) { s3[0] += part[3 * t]; s3[1] += part[3 * t + 1]; s3[2] += part[3 * t + 2]; }
    free(part);
}

static double canonical(const double* s3, double eta, double omega) {
    double v = (omega / eta) * s3[0] + (1.0 / (eta * omega)) * s3[1] - 2.0 * s3[2];
    return sqrt(v > 0.0 ? v : 0.0);
}

typedef struct { double primal, dual, gap; } Gap;

/* Primal (upper) bound sum_{i,s} K_i max_{t>=s} x + sum_s K0 max_{i,t>=s} x
 * + <H, x>, dual (lower) bound sum_{i,t} min_{s<=t} (h + y + z), both at the
 * original scale. */
static Gap gap_at(const Shape* d, const Trio* st) {
    double term1 = 0, term2 = 0, term3 = 0, dual = 0;
    for (int64_t i = 0; i < d->n; ++i)
        for (int64_t s = 0; s < d->tp; ++s) {
            double mx = -INFINITY;
            for (int64_t t = s; t < d->tp; ++t) mx = fmax(mx, d->k[i] * st->x[at(d, i, s, t)]);
            term1 += mx;
        }
    for (int64_t s = 0; s < d->tp; ++s) {
        double mx = -INFINITY;
        for (int64_t i = 0; i < d->n; ++i)
            for (int64_t t = s; t < d->tp; ++t) mx = fmax(mx, d->k0 * st->x[at(d, i, s, t)]);
        term2 += mx;
    }
    for (int64_t g = 0; g < d->ND; ++g) term3 += st->x[g] * d->h[g];
    for (int64_t i = 0; i < d->n; ++i)
        for (int64_t t = 0; t < d->tp; ++t) {
            double mn = INFINITY;
            for (int64_t s = 0; s <= t; ++s) {
                int64_t g = at(d, i, s, t);
                mn = fmin(mn, d->h[g] + st->y[g] + st->z[g]);
            }
            dual += mn;
        }
    Gap r;
    r.primal = (term1 + term2 + term3) * d->scale;
    r.dual = dual * d->scale;
    r.gap = (r.primal - r.dual) / (1.0 + fabs(r.dual) + fabs(r.primal));
    return r;
}

static int keep_going(double gap, int64_t iteration, int64_t max_iter, double tol) {
    int within = iteration < max_iter || max_iter < 0;
    return within && !(gap <= tol);
}

/* Objective of a primal x on the ORIGINAL [n][t][t] problem
 * (jrp/pria-jax/pria/jrp_problem.py:143-161): the maxima run over whole rows. */
ORACLE_EXPORT double oracle_pria_objective(int64_t n, int64_t t, const double* k, double k0,
                                           const double* h, const double* x) {
    double obj = 0.0;
    for (int64_t i = 0; i < n; ++i)
        for (int64_t s = 0; s < t; ++s) {
            double mx = 0.0;
            for (int64_t tt = 0; tt < t; ++tt) mx = fmax(mx, x[(i * t + s) * t + tt]);
            obj += k[i] * mx;
        }
    for (int64_t s = 0; s < t; ++s) {
        double mx = 0.0;
        for (int64_t i = 0; i < n; ++i)
            for (int64_t tt = 0; tt < t; ++tt) mx = fmax(mx, x[(i * t + s) * t + tt]);
        obj += k0 * mx;
    }
    for (int64_t i = 0; i < n; ++i)
        for (int64_t s = 0; s < t; ++s)
            for (int64_t tt = s; tt < t; ++tt)
                obj += h[(i * t + s) * t + tt] * x[(i * t + s) * t + tt];
    return obj;
}

/* Solve.  H is dense row-major [n][t][t] (upper triangle read).  Outputs
 * x, y, z (each [n][t][t] or NULL) use the normalised dual convention: y / K_i,
 * z / K0.  out[0..4) = iterations, primal (upper, at the unpadded x),
 * dual (lower, the padded dual bound the solver converged against),
 * relative gap of those two.  Returns 0, or -1 for a bad argument. */
ORACLE_EXPORT int oracle_pria_solve(int64_t n, int64_t t, const double* K, double K0,
                                    const double* H, const OraclePriaParams* params,
                                    int threads, double* xo, double* yo, double* zo,
                                    double* out) {
    out[0] = 0; out[1] = out[2] = out[3] = NAN;
    if (n < 1 || t < 1 || !K || !H || !params) return -1;
    OraclePriaParams p = *params;
    if (p.op_steps < 2) p.op_steps = 2;
    if (p.warm_steps < 0) p.warm_steps = 0;

    Shape d;
    d.n = n; d.t = t; d.tp = t + (t & 1);
    d.P = d.tp * (d.tp + 1) / 2;
    d.ND = n * d.P;
    d.threads = threads;
    double ss = K0 * K0;
    for (int64_t i = 0; i < n; ++i) ss += K[i] * K[i];
    for (int64_t i = 0; i < n; ++i)
        for (int64_t s = 0; s < t; ++s)
            for (int64_t tt = s; tt < t; ++tt) {
                double v = H[(i * t + s) * t + tt];
                ss += v * v;
            }
    d.scale = ss > 0.0 ? sqrt(ss) : 1.0;
    d.k = (double*)malloc(sizeof(double) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) d.k[i] = K[i] / d.scale;
    d.k0 = K0 / d.scale;
    d.h = (double*)calloc((size_t)d.ND, sizeof(double));
    for (int64_t i = 0; i < n; ++i)
        for (int64_t s = 0; s < t; ++s)
            for (int64_t tt = s; tt < t; ++tt) d.h[at(&d, i, s, tt)] = H[(i * t + s) * t + tt] / d.scale;

    Trio cur, step, anchor, next;
    trio_alloc(&cur, d.ND); trio_alloc(&step, d.ND); trio_alloc(&anchor, d.ND); trio_alloc(&next, d.ND);
    proj_x(&d, cur.x);
    proj_y(&d, cur.y);
    proj_z(&d, cur.z);
    trio_copy(&anchor, &cur, d.ND);
    double omega = p.omega, eta = p.eta;
    int64_t iteration = 0;
    raw_step(&d, omega, eta, &cur, &step);
    Gap gi = {0.0, 0.0, INFINITY};

    /* The vanilla phase: warm_steps blocks with Halpern, or the whole solve
     * without it.  With the defaults (warm_steps 0) it does nothing. */
    int64_t warm_budget = p.use_halpern ? (int64_t)p.op_steps * p.warm_steps : p.max_iter;
    if (!p.use_halpern || warm_budget != 0) {
        for (;;) {
            gi = gap_at(&d, &cur);
            if (!keep_going(gi.gap, iteration, warm_budget, p.tolerance)) break;
            for (int k = 0; k < p.op_steps; ++k) {
                raw_step(&d, omega, eta, &step, &next);
                Trio tmp = cur; cur = step; step = next; next = tmp;
                ++iteration;
            }
        }
    }
    if (iteration > 0) {
        double s3[3];
        diffs(&d, &cur, &anchor, s3);
        double om = sqrt(s3[1]) / sqrt(s3[0]);
        omega = isnan(om) ? p.omega : om;
    }

    int report_step = 0;
    if (p.use_halpern) {
        double theta = p.theta_initial, check_err = INFINITY;
        int64_t restart_iter = 0;
        trio_copy(&anchor, &cur, d.ND);
        double s3[3];
        diffs(&d, &cur, &step, s3);
        double fp_err = canonical(s3, eta, omega);
        gi = gap_at(&d, &cur);
        int terminated = !keep_going(gi.gap, iteration, p.max_iter, p.tolerance);
        while (!terminated) {
            report_step = 1;
            for (int k = 0; k < p.op_steps; ++k) {
                double lw = (double)(restart_iter + 1) / (double)(restart_iter + 2);
                double rw = 1.0 / (double)(restart_iter + 2);
#pragma omp parallel for schedule(static) num_threads(nth(&d))
                for (int64_t g = 0; g < d.ND; ++g) {
                    cur.x[g] = lw * (2.0 * step.x[g] - cur.x[g]) + rw * anchor.x[g];
                    cur.y[g] = lw * (2.0 * step.y[g] - cur.y[g]) + rw * anchor.y[g];
                    cur.z[g] = lw * (2.0 * step.z[g] - cur.z[g]) + rw * anchor.z[g];
                }
                raw_step(&d, omega, eta, &cur, &step);
                ++restart_iter;
                ++iteration;
            }
            diffs(&d, &cur, &step, s3);
            double new_err = canonical(s3, eta, omega);
            gi = gap_at(&d, &step);
            terminated = !keep_going(gi.gap, iteration, p.max_iter, p.tolerance);
            int sufficient = new_err <= p.beta_sufficient * fp_err;
            int necessary = new_err <= p.beta_necessary * fp_err && new_err > check_err;
            int artificial = (double)restart_iter >= p.beta_artificial * (double)iteration;
            if (terminated) break;
            if (sufficient || necessary || artificial) {
                double d3[3];
                diffs(&d, &cur, &anchor, d3);
                double pn = sqrt(d3[0]), dn = sqrt(d3[1]);
                if (pn > 1e-16 && dn > 1e-16) {
                    omega = exp(theta * (log(dn) - log(pn)) + (1.0 - theta) * log(omega));
                    theta = p.theta_target + p.theta_decay * (theta - p.theta_target);
                }
                trio_copy(&anchor, &step, d.ND);
                raw_step(&d, omega, eta, &step, &next);
                Trio tmp = cur; cur = step; step = next; next = tmp;
                diffs(&d, &cur, &step, s3);
                fp_err = canonical(s3, eta, omega);
                check_err = INFINITY;
                restart_iter = 0;
            } else {
                check_err = new_err;
            }
        }
    }

    const Trio* fin = report_step ? &step : &cur;
    double* xfull = xo ? xo : (double*)malloc(sizeof(double) * (size_t)(n * t * t));
    memset(xfull, 0, sizeof(double) * (size_t)(n * t * t));
    if (yo) memset(yo, 0, sizeof(double) * (size_t)(n * t * t));
    if (zo) memset(zo, 0, sizeof(double) * (size_t)(n * t * t));
    for (int64_t i = 0; i < n; ++i)
        for (int64_t s = 0; s < t; ++s)
            for (int64_t tt = s; tt < t; ++tt) {
                int64_t g = at(&d, i, s, tt), go = (i * t + s) * t + tt;
                xfull[go] = fin->x[g];
                if (yo) yo[go] = d.k[i] > 0.0 ? fin->y[g] / d.k[i] : 0.0;
                if (zo) zo[go] = d.k0 > 0.0 ? fin->z[g] / d.k0 : 0.0;
            }
    double upper = oracle_pria_objective(n, t, K, K0, H, xfull);
    out[0] = (double)iteration;
    out[1] = upper;
    out[2] = gi.dual;
    out[3] = (upper - gi.dual) / (1.0 + fabs(upper) + fabs(gi.dual));
    if (!xo) free(xfull);
    trio_free(&cur); trio_free(&step); trio_free(&anchor); trio_free(&next);
    free(d.k); free(d.h);
    return 0;
}
