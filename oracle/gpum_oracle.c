/*
 * gpum_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement, in f64, of the reference's native CPU backend
 * (src/rust/src/cpu_native.rs of pcbrom/gpumetropolis 0.7.0).  It is the
 * checker for the B200 path and the timed CPU baseline; only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.  The
 * product path never calls it.
 *
 * The reference itself (Rust + extendr + Cranelift) cannot be built here, so
 * this port is pinned against the known answers held by the reference's own
 * tests (tests/testthat/test-dsl.R, test-catalog.R, test-mala.R,
 * test-kernel.R, test-adaptive.R) plus closed-form posteriors; see
 * tests/golden/.
 *
 * Every function follows one reference function; the arithmetic order is kept
 * so results match the reference's f64 path to the last bit where the
 * platform libm is the same (glibc exp/log/pow/sqrt/cos).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define GPO_STACK 32

/* triple32 integer hash (cpu_native.rs:14-23). */
uint32_t gpo_triple32(uint32_t h) {
    h ^= h >> 17;
    h *= 2129725213u;
    h ^= h >> 11;
    h *= 2890025505u;
    h ^= h >> 15;
    h *= 831628273u;
    h ^= h >> 14;
    return h;
}

/* One uniform in (0,1) from a counter (cpu_native.rs:26-28). */
double gpo_uniform(uint32_t seedmix, uint32_t ctr) {
    return ((double)gpo_triple32(seedmix + ctr) + 0.5) / 4294967296.0;
}

/* Per-chain stream offset: hash of the seed plus chain * golden-ratio
 * constant, wrapping (cpu_native.rs:561-562). */
uint32_t gpo_seedmix(uint32_t seed, uint32_t chain) {
    return gpo_triple32(seed) + chain * 2654435761u;
}

/* Log-gamma, Lanczos with g = 7 and the nine published coefficients, with
 * the reflection formula below 0.5 (cpu_native.rs:34-60). */
double gpo_lgamma(double x) {
    static const double c[9] = {
        0.99999999999980993, 676.5203681218851, -1259.1392167224028,
        771.32342877765313, -176.61502916214059, 12.507343278686905,
        -0.13857109526572012, 9.9843695780195716e-6, 1.5056327351493116e-7};
    const double pi = 3.141592653589793;
    if (x < 0.5) {
        return log(fabs(pi / sin(pi * x))) - gpo_lgamma(1.0 - x);
    }
    double xm = x - 1.0;
    double a = c[0];
    double t = xm + 7.0 + 0.5;
    for (int i = 1; i < 9; ++i) a += c[i] / (xm + (double)i);
    return 0.5 * log(2.0 * pi) + (xm + 0.5) * log(t) - t + log(a);
}

/* Digamma: recurrence up past 6, then the asymptotic series
 * (cpu_native.rs:66-77). */
double gpo_digamma(double x) {
    double r = 0.0;
    while (x < 6.0) {
        r -= 1.0 / x;
        x += 1.0;
    }
    double f = 1.0 / (x * x);
    return r + log(x) - 1.0 / (2.0 * x)
           - f * (1.0 / 12.0 - f * (1.0 / 120.0 - f * (1.0 / 252.0)));
}

/* Interpret one program on one observation row (cpu_native.rs:80-107).
 * Empty program -> 0; every opcode outside {0..10,12} acts as POW. */
double gpo_eval(const uint32_t *code, size_t n_instr, const double *consts,
                const double *params, const double *row) {
    if (n_instr == 0) return 0.0;
    double st[GPO_STACK];
    size_t sp = 0;
    for (size_t pc = 0; pc < n_instr; ++pc) {
        uint32_t op = code[2 * pc], arg = code[2 * pc + 1];
        switch (op) {
        case 0: st[sp++] = consts[arg]; break;
        case 1: st[sp++] = params[arg]; break;
        case 2: st[sp++] = row[arg]; break;
        case 3: st[sp - 2] += st[sp - 1]; sp--; break;
        case 4: st[sp - 2] -= st[sp - 1]; sp--; break;
        case 5: st[sp - 2] *= st[sp - 1]; sp--; break;
        case 6: st[sp - 2] /= st[sp - 1]; sp--; break;
        case 7: st[sp - 1] = -st[sp - 1]; break;
        case 8: st[sp - 1] = exp(st[sp - 1]); break;
        case 9: st[sp - 1] = log(st[sp - 1]); break;
        case 10: st[sp - 1] = sqrt(st[sp - 1]); break;
        case 12: st[sp - 1] = gpo_lgamma(st[sp - 1]); break;
        default: st[sp - 2] = pow(st[sp - 2], st[sp - 1]); sp--; break;
        }
    }
    return st[0];
}

/* Data-term sum over observations, sequential f64 accumulation
 * (cpu_native.rs:110-117; the JIT path jit.rs:512-604 sums in the same
 * order). */
double gpo_loglik_sum(const uint32_t *code, size_t n_instr, const double *consts,
                      const double *params, const double *data, size_t n_cols,
                      size_t n_obs) {
    double acc = 0.0;
    for (size_t i = 0; i < n_obs; ++i)
        acc += gpo_eval(code, n_instr, consts, params, data + i * n_cols);
    return acc;
}

/* Reverse-mode tape for one program at one row (cpu_native.rs:148-279).
 * `grad` is accumulated into, not overwritten.  Scratch arrays are sized
 * n_instr by the caller. */
typedef struct {
    double *vals, *adj;
    uint32_t *lhs, *rhs;
} gpo_tape;

static double gpo_eval_grad(const uint32_t *code, size_t n_instr,
                            const double *consts, const double *params,
                            const double *row, gpo_tape *w, double *grad) {
    if (n_instr == 0) return 0.0;
    uint32_t ist[GPO_STACK];
    size_t sp = 0;
    for (size_t pc = 0; pc < n_instr; ++pc) {
        uint32_t op = code[2 * pc], arg = code[2 * pc + 1];
        if (op <= 2) {
            w->vals[pc] = op == 0 ? consts[arg] : (op == 1 ? params[arg] : row[arg]);
            w->lhs[pc] = UINT32_MAX;
            ist[sp++] = (uint32_t)pc;
        } else if ((op >= 7 && op <= 10) || op == 12) {
            uint32_t l = ist[sp - 1];
            double x = w->vals[l];
            double v;
            switch (op) {
            case 7: v = -x; break;
            case 8: v = exp(x); break;
            case 9: v = log(x); break;
            case 10: v = sqrt(x); break;
            default: v = gpo_lgamma(x); break;
            }
            w->vals[pc] = v;
            w->lhs[pc] = l;
            w->rhs[pc] = UINT32_MAX;
            ist[sp - 1] = (uint32_t)pc;
        } else {
            uint32_t r = ist[sp - 1], l = ist[sp - 2];
            double a = w->vals[l], b = w->vals[r], v;
            switch (op) {
            case 3: v = a + b; break;
            case 4: v = a - b; break;
            case 5: v = a * b; break;
            case 6: v = a / b; break;
            default: v = pow(a, b); break;
            }
            w->vals[pc] = v;
            w->lhs[pc] = l;
            w->rhs[pc] = r;
            ist[sp - 2] = (uint32_t)pc;
            sp--;
        }
    }
    size_t root = n_instr - 1;
    for (size_t i = 0; i < n_instr; ++i) w->adj[i] = 0.0;
    w->adj[root] = 1.0;
    for (size_t k = n_instr; k-- > 0;) {
        double g = w->adj[k];
        if (g == 0.0) continue;
        uint32_t op = code[2 * k], arg = code[2 * k + 1];
        uint32_t l = w->lhs[k], r = w->rhs[k];
        switch (op) {
        case 0: case 2: break;
        case 1: grad[arg] += g; break;
        case 3: w->adj[l] += g; w->adj[r] += g; break;
        case 4: w->adj[l] += g; w->adj[r] -= g; break;
        case 5: w->adj[l] += g * w->vals[r]; w->adj[r] += g * w->vals[l]; break;
        case 6:
            w->adj[l] += g / w->vals[r];
            w->adj[r] -= g * w->vals[k] / w->vals[r];
            break;
        case 7: w->adj[l] -= g; break;
        case 8: w->adj[l] += g * w->vals[k]; break;
        case 9: w->adj[l] += g / w->vals[l]; break;
        case 10: w->adj[l] += g * 0.5 / w->vals[k]; break;
        case 12: w->adj[l] += g * gpo_digamma(w->vals[l]); break;
        default: {
            double a = w->vals[l], b = w->vals[r];
            w->adj[l] += g * b * pow(a, b - 1.0);
            if (a > 0.0) w->adj[r] += g * w->vals[k] * log(a);
            break;
        }
        }
    }
    return w->vals[root];
}

static int gpo_tape_alloc(gpo_tape *w, size_t n) {
    if (n < 1) n = 1;
    w->vals = (double *)malloc(n * sizeof(double));
    w->adj = (double *)malloc(n * sizeof(double));
    w->lhs = (uint32_t *)malloc(n * sizeof(uint32_t));
    w->rhs = (uint32_t *)malloc(n * sizeof(uint32_t));
    return (w->vals && w->adj && w->lhs && w->rhs) ? 0 : -1;
}

static void gpo_tape_free(gpo_tape *w) {
    free(w->vals); free(w->adj); free(w->lhs); free(w->rhs);
}

/* Value of the summed data term and its gradient, zeroing grad first
 * (the data half of cpu_native.rs:285-298, which grad_batch :306-329 also
 * uses).  Returns the value. */
double gpo_loglik_grad(const uint32_t *code, size_t n_instr, const double *consts,
                       size_t n_params, const double *params, const double *data,
                       size_t n_cols, size_t n_obs, double *grad) {
    gpo_tape w;
    if (gpo_tape_alloc(&w, n_instr) != 0) return NAN;
    for (size_t j = 0; j < n_params; ++j) grad[j] = 0.0;
    double acc = 0.0;
    for (size_t i = 0; i < n_obs; ++i)
        acc += gpo_eval_grad(code, n_instr, consts, params, data + i * n_cols, &w, grad);
    gpo_tape_free(&w);
    return acc;
}

/* Log-likelihood at each point (cpu_native.rs:339-360). */
void gpo_loglik_batch(const uint32_t *code, size_t n_instr, const double *consts,
                      size_t n_params, const double *data, size_t n_cols, size_t n_obs,
                      const double *points, size_t n_points, double *out) {
#pragma omp parallel for schedule(dynamic)
    for (long p = 0; p < (long)n_points; ++p)
        out[p] = gpo_loglik_sum(code, n_instr, consts, points + p * n_params, data,
                                n_cols, n_obs);
}

/* Gradient of the data term at each point, point-major (cpu_native.rs:306-329). */
void gpo_grad_batch(const uint32_t *code, size_t n_instr, const double *consts,
                    size_t n_params, const double *data, size_t n_cols, size_t n_obs,
                    const double *points, size_t n_points, double *out) {
#pragma omp parallel for schedule(dynamic)
    for (long p = 0; p < (long)n_points; ++p)
        gpo_loglik_grad(code, n_instr, consts, n_params, points + p * n_params, data,
                        n_cols, n_obs, out + p * n_params);
}

/* Per-observation log-likelihood, out[p * n_obs + i] (cpu_native.rs:371-391). */
void gpo_loglik_pointwise(const uint32_t *code, size_t n_instr, const double *consts,
                          size_t n_params, const double *data, size_t n_cols,
                          size_t n_obs, const double *points, size_t n_points,
                          double *out) {
#pragma omp parallel for schedule(dynamic)
    for (long p = 0; p < (long)n_points; ++p)
        for (size_t i = 0; i < n_obs; ++i)
            out[p * n_obs + i] = gpo_eval(code, n_instr, consts, points + p * n_params,
                                          data + i * n_cols);
}

/* A compiled data-term evaluator (the jit.rs analogue): same contract as
 * gpo_loglik_sum for one parameter vector. */
typedef double (*gpo_loglik_fn)(const double *params, const double *data,
                                int64_t n_obs, int64_t n_cols);

/* Checker at full configuration sizes (not a reference function): the
 * compiled evaluator `fn` at each point, parallel over points.  With the
 * evaluator cjit emits, the result is gpo_loglik_batch's value (same f64
 * operations in the same order). */
void gpo_jit_batch(gpo_loglik_fn fn, size_t n_params, const double *data, size_t n_cols,
                   size_t n_obs, const double *points, size_t n_points, double *out,
                   int n_threads) {
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic) num_threads(n_threads)
    for (long p = 0; p < (long)n_points; ++p)
        out[p] = fn(points + p * n_params, data, (int64_t)n_obs, (int64_t)n_cols);
}

/* Checker at full configuration sizes (not a reference function): the
 * data-term gradient of cpu_native.rs:306-329 at each point, and per
 * component the sum over observations of the per-observation gradient's
 * absolute value (the scale a cancelling sum's rounding error is bounded
 * by).  Parallel over (point, block of `block` observations); the blocks of
 * a point are added in block order.  out_grad, out_abs: point-major. */
int gpo_grad_abs_batch(const uint32_t *code, size_t n_instr, const double *consts,
                       size_t n_params, const double *data, size_t n_cols, size_t n_obs,
                       const double *points, size_t n_points, size_t block,
                       double *out_grad, double *out_abs, int n_threads) {
    if (n_threads <= 0) n_threads = omp_get_max_threads();
    if (block < 1) block = 1;
    const size_t nb = n_obs ? (n_obs + block - 1) / block : 1;
    double *part = (double *)calloc(n_points * nb * 2 * (n_params ? n_params : 1),
                                    sizeof(double));
    if (!part) return -1;
    int err = 0;
#pragma omp parallel num_threads(n_threads) reduction(| : err)
    {
        gpo_tape w;
        double *g1 = (double *)malloc((n_params ? n_params : 1) * sizeof(double));
        const int ok = gpo_tape_alloc(&w, n_instr) == 0 && g1 != NULL;
        if (!ok) err = 1;
        /* every thread reaches the worksharing loop; one without scratch skips */
#pragma omp for schedule(dynamic)
            for (long t = 0; t < (long)(n_points * nb); ++t) {
                if (!ok) continue;
                const size_t p = (size_t)t / nb, b = (size_t)t % nb;
                double *pg = part + (size_t)t * 2 * n_params, *pa = pg + n_params;
                const size_t i1 = (b + 1) * block < n_obs ? (b + 1) * block : n_obs;
                for (size_t i = b * block; i < i1; ++i) {
                    for (size_t j = 0; j < n_params; ++j) g1[j] = 0.0;
                    gpo_eval_grad(code, n_instr, consts, points + p * n_params,
                                  data + i * n_cols, &w, g1);
                    for (size_t j = 0; j < n_params; ++j) {
                        pg[j] += g1[j];
                        pa[j] += fabs(g1[j]);
                    }
                }
            }
        gpo_tape_free(&w);
        free(g1);
    }
    for (size_t p = 0; p < n_points; ++p)
        for (size_t j = 0; j < n_params; ++j) {
            double sg = 0.0, sa = 0.0;
            for (size_t b = 0; b < nb; ++b) {
                sg += part[((p * nb + b) * 2) * n_params + j];
                sa += part[((p * nb + b) * 2 + 1) * n_params + j];
            }
            out_grad[p * n_params + j] = sg;
            out_abs[p * n_params + j] = sa;
        }
    free(part);
    return err ? -1 : 0;
}

typedef struct {
    const uint32_t *code; size_t n_instr; const double *consts;
    const uint32_t *prior_code; size_t n_prior; const double *prior_consts;
    size_t n_params; const double *data; size_t n_cols; size_t n_obs;
    gpo_loglik_fn jit;
} gpo_model;

static double gpo_log_post(const gpo_model *m, const double *params) {
    double ll = m->jit ? m->jit(params, m->data, (int64_t)m->n_obs, (int64_t)m->n_cols)
                       : gpo_loglik_sum(m->code, m->n_instr, m->consts, params, m->data,
                                        m->n_cols, m->n_obs);
    return ll + gpo_eval(m->prior_code, m->n_prior, m->prior_consts, params, NULL);
}

/* Value and gradient of the log posterior, grad overwritten
 * (cpu_native.rs:285-298 / :589-602). */
static double gpo_log_post_grad(const gpo_model *m, const double *params,
                                gpo_tape *w, double *grad) {
    for (size_t j = 0; j < m->n_params; ++j) grad[j] = 0.0;
    double acc = 0.0;
    for (size_t i = 0; i < m->n_obs; ++i)
        acc += gpo_eval_grad(m->code, m->n_instr, m->consts, params,
                             m->data + i * m->n_cols, w, grad);
    return acc + gpo_eval_grad(m->prior_code, m->n_prior, m->prior_consts, params,
                               NULL, w, grad);
}

static inline double gpo_normal(uint32_t seedmix, uint32_t *ctr) {
    const double two_pi = 6.283185307179586;
    *ctr += 1;
    double u1 = gpo_uniform(seedmix, *ctr);
    *ctr += 1;
    double u2 = gpo_uniform(seedmix, *ctr);
    return sqrt(-2.0 * log(u1)) * cos(two_pi * u2);
}

/* out = f * (1/2) M g with M = Ls Ls' (or diag sd^2), the drift capped at a
 * whitened norm of 2 sqrt(d) (cpu_native.rs:617-651). */
static void gpo_half_m_times(size_t np, const double *sd, const double *L,
                             const double *g, double *out, double *tmp) {
    double drift_max = 2.0 * sqrt((double)np);
    if (!L) {
        for (size_t j = 0; j < np; ++j) tmp[j] = 0.5 * sd[j] * g[j];
    } else {
        for (size_t j = 0; j < np; ++j) {
            double acc = 0.0;
            for (size_t k = j; k < np; ++k) acc += L[k * np + j] * g[k];
            tmp[j] = 0.5 * acc;
        }
    }
    double ss = 0.0;
    for (size_t j = 0; j < np; ++j) ss += tmp[j] * tmp[j];
    double norm = sqrt(ss);
    double f = norm > drift_max ? drift_max / norm : 1.0;
    if (!L) {
        for (size_t j = 0; j < np; ++j) out[j] = f * sd[j] * tmp[j];
    } else {
        for (size_t k = 0; k < np; ++k) {
            double acc = 0.0;
            for (size_t j = 0; j <= k; ++j) acc += L[k * np + j] * tmp[j];
            out[k] = f * acc;
        }
    }
}

/* -1/2 |Ls^{-1}(v - m)|^2 (cpu_native.rs:655-673). */
static double gpo_log_q(size_t np, const double *sd, const double *L, const double *v,
                        const double *m, double *tmp) {
    double q = 0.0;
    if (!L) {
        for (size_t j = 0; j < np; ++j) {
            double r = (v[j] - m[j]) / sd[j];
            q -= 0.5 * r * r;
        }
    } else {
        for (size_t k = 0; k < np; ++k) {
            double acc = v[k] - m[k];
            for (size_t j = 0; j < k; ++j) acc -= L[k * np + j] * tmp[j];
            tmp[k] = acc / L[k * np + k];
            q -= 0.5 * tmp[k] * tmp[k];
        }
    }
    return q;
}

/* Whole-chain sampler, parallel over chains (cpu_native.rs:510-825).
 * proposal_mode: 0 diagonal RWM, 2 Cholesky RWM, 3 MALA, anything else DE.
 * proposal_l is NULL or n_chains*np*np chain-major row-major lower factors.
 * draws: f32, column-major (n_iter, n_chains, np).  n_threads <= 0: all. */
int gpo_run(const uint32_t *code, size_t n_instr, const double *consts,
            const uint32_t *prior_code, size_t n_prior, const double *prior_consts,
            size_t np, const double *data, size_t n_cols, size_t n_obs,
            const double *init, const double *proposal_sd, const double *temperatures,
            size_t n_chains, size_t n_iter, uint32_t seed, uint32_t mode,
            double gamma, double de_noise, const double *proposal_l,
            gpo_loglik_fn jit, int n_threads,
            float *out_draws, float *out_accept, double *out_last) {
    gpo_model m = {code, n_instr, consts, prior_code, n_prior, prior_consts,
                   np, data, n_cols, n_obs, jit};
    int err = 0;
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#else
    (void)n_threads;
#endif
#pragma omp parallel for schedule(dynamic) num_threads(n_threads) reduction(| : err)
    for (long cl = 0; cl < (long)n_chains; ++cl) {
        size_t c = (size_t)cl, pb = c * np;
        double temp = temperatures[c];
        uint32_t seedmix = gpo_seedmix(seed, (uint32_t)c);
        const double *sd = proposal_sd + pb;
        const double *L = proposal_l ? proposal_l + c * np * np : NULL;
        size_t nt = n_instr > n_prior ? n_instr : n_prior;
        double *buf = (double *)malloc(9 * (np + 1) * sizeof(double));
        gpo_tape w;
        if (!buf || gpo_tape_alloc(&w, nt) != 0) { err |= 1; free(buf); continue; }
        double *state = buf, *prop = buf + (np + 1), *z = buf + 2 * (np + 1);
        double *gx = buf + 3 * (np + 1), *gy = buf + 4 * (np + 1);
        double *mx = buf + 5 * (np + 1), *my = buf + 6 * (np + 1);
        double *vb = buf + 7 * (np + 1);
        memcpy(state, init + pb, np * sizeof(double));
        memcpy(prop, state, np * sizeof(double));
        int mala = mode == 3;
        double cur = mala ? gpo_log_post_grad(&m, state, &w, gx) : gpo_log_post(&m, state);
        uint32_t ctr = 0, acc = 0;
        for (size_t t = 0; t < n_iter; ++t) {
            if (mala) {
                gpo_half_m_times(np, sd, L, gx, mx, vb);
                for (size_t j = 0; j < np; ++j) {
                    mx[j] += state[j];
                    z[j] = gpo_normal(seedmix, &ctr);
                }
                if (!L) {
                    for (size_t j = 0; j < np; ++j) prop[j] = mx[j] + sd[j] * z[j];
                } else {
                    for (size_t k = 0; k < np; ++k) {
                        double a = mx[k];
                        for (size_t j = 0; j <= k; ++j) a += L[k * np + j] * z[j];
                        prop[k] = a;
                    }
                }
                double plp = gpo_log_post_grad(&m, prop, &w, gy);
                gpo_half_m_times(np, sd, L, gy, my, vb);
                for (size_t j = 0; j < np; ++j) my[j] += prop[j];
                double lqd = gpo_log_q(np, sd, L, state, my, vb)
                             - gpo_log_q(np, sd, L, prop, mx, vb);
                ctr += 1;
                double u = gpo_uniform(seedmix, ctr);
                if (isfinite(plp) && log(u) < (plp - cur) / temp + lqd) {
                    memcpy(state, prop, np * sizeof(double));
                    double *tg = gx; gx = gy; gy = tg;
                    cur = plp;
                    acc++;
                }
            } else {
                if (mode == 0) {
                    for (size_t j = 0; j < np; ++j)
                        prop[j] = state[j] + sd[j] * gpo_normal(seedmix, &ctr);
                } else if (mode == 2) {
                    for (size_t j = 0; j < np; ++j) z[j] = gpo_normal(seedmix, &ctr);
                    for (size_t k = 0; k < np; ++k) {
                        double a = state[k];
                        for (size_t j = 0; j <= k; ++j) a += L[k * np + j] * z[j];
                        prop[k] = a;
                    }
                } else {
                    ctr += 1;
                    size_t a = (size_t)(gpo_uniform(seedmix, ctr) * (double)n_chains);
                    if (a >= n_chains) a = n_chains - 1;
                    ctr += 1;
                    size_t b = (size_t)(gpo_uniform(seedmix, ctr) * (double)n_chains);
                    if (b >= n_chains) b = n_chains - 1;
                    if (b == a) b = (b + 1) % n_chains;
                    ctr += 1;
                    double g = gpo_uniform(seedmix, ctr) < 0.1 ? 1.0 : gamma;
                    for (size_t j = 0; j < np; ++j) {
                        double zz = gpo_normal(seedmix, &ctr);
                        double diff = init[a * np + j] - init[b * np + j];
                        prop[j] = state[j] + g * diff + de_noise * sd[j] * zz;
                    }
                }
                double plp = gpo_log_post(&m, prop);
                ctr += 1;
                double u = gpo_uniform(seedmix, ctr);
                if (log(u) < (plp - cur) / temp) {
                    memcpy(state, prop, np * sizeof(double));
                    cur = plp;
                    acc++;
                }
            }
            for (size_t j = 0; j < np; ++j)
                out_draws[t + n_iter * (c + n_chains * j)] = (float)state[j];
        }
        out_accept[c] = n_iter == 0 ? 0.0f : (float)acc / (float)n_iter;
        out_last[c] = cur;
        gpo_tape_free(&w);
        free(buf);
    }
    return err ? -1 : 0;
}

/* Synchronous per-generation DE, pair excludes self (cpu_native.rs:400-506). */
int gpo_run_de_sync(const uint32_t *code, size_t n_instr, const double *consts,
                    const uint32_t *prior_code, size_t n_prior,
                    const double *prior_consts, size_t np, const double *data,
                    size_t n_cols, size_t n_obs, const double *init,
                    const double *proposal_sd, size_t n_chains, size_t n_iter,
                    uint32_t seed, double gamma, double de_noise, gpo_loglik_fn jit,
                    float *out_draws, float *out_accept, double *out_last) {
    gpo_model m = {code, n_instr, consts, prior_code, n_prior, prior_consts,
                   np, data, n_cols, n_obs, jit};
    size_t nn = n_chains * np;
    double *cur_pop = (double *)malloc(nn * sizeof(double));
    double *nxt_pop = (double *)malloc(nn * sizeof(double));
    double *lp = (double *)malloc(n_chains * sizeof(double));
    double *lp_next = (double *)malloc(n_chains * sizeof(double));
    uint32_t *ctrs = (uint32_t *)calloc(n_chains, sizeof(uint32_t));
    uint32_t *accs = (uint32_t *)calloc(n_chains, sizeof(uint32_t));
    double *props = (double *)malloc(nn * sizeof(double));
    if (!cur_pop || !nxt_pop || !lp || !lp_next || !ctrs || !accs || !props) {
        free(cur_pop); free(nxt_pop); free(lp); free(lp_next); free(ctrs); free(accs);
        free(props);
        return -1;
    }
    memcpy(cur_pop, init, nn * sizeof(double));
#pragma omp parallel for schedule(dynamic)
    for (long c = 0; c < (long)n_chains; ++c) lp[c] = gpo_log_post(&m, cur_pop + c * np);
    for (size_t t = 0; t < n_iter; ++t) {
#pragma omp parallel for schedule(dynamic)
        for (long cl = 0; cl < (long)n_chains; ++cl) {
            size_t c = (size_t)cl, pb = c * np;
            uint32_t seedmix = gpo_seedmix(seed, (uint32_t)c);
            uint32_t ctr = ctrs[c];
            const double *state = cur_pop + pb;
            double *prop = props + pb;
            ctr += 1;
            size_t a = (size_t)(gpo_uniform(seedmix, ctr) * (double)n_chains);
            if (a >= n_chains) a = n_chains - 1;
            if (a == c) a = (a + 1) % n_chains;
            ctr += 1;
            size_t b = (size_t)(gpo_uniform(seedmix, ctr) * (double)n_chains);
            if (b >= n_chains) b = n_chains - 1;
            while (b == c || b == a) b = (b + 1) % n_chains;
            ctr += 1;
            double g = gpo_uniform(seedmix, ctr) < 0.1 ? 1.0 : gamma;
            for (size_t j = 0; j < np; ++j) {
                double zz = gpo_normal(seedmix, &ctr);
                double diff = cur_pop[a * np + j] - cur_pop[b * np + j];
                prop[j] = state[j] + g * diff + de_noise * proposal_sd[pb + j] * zz;
            }
            double plp = gpo_log_post(&m, prop);
            ctr += 1;
            double u = gpo_uniform(seedmix, ctr);
            int take = log(u) < plp - lp[c];
            memcpy(nxt_pop + pb, take ? prop : state, np * sizeof(double));
            lp_next[c] = take ? plp : lp[c];
            ctrs[c] = ctr;
            if (take) accs[c]++;
        }
        for (size_t c = 0; c < n_chains; ++c)
            for (size_t j = 0; j < np; ++j)
                out_draws[t + n_iter * (c + n_chains * j)] = (float)nxt_pop[c * np + j];
        double *tp = cur_pop; cur_pop = nxt_pop; nxt_pop = tp;
        double *tl = lp; lp = lp_next; lp_next = tl;
    }
    for (size_t c = 0; c < n_chains; ++c) {
        out_accept[c] = n_iter == 0 ? 0.0f : (float)accs[c] / (float)n_iter;
        out_last[c] = lp[c];
    }
    free(cur_pop); free(nxt_pop); free(lp); free(lp_next); free(ctrs); free(accs);
    free(props);
    return 0;
}
