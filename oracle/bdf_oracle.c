/*
 * bdf_oracle.c -- FP64 host oracle for the time-varying CME path (dp/dt = A(t) p).
 *
 * TEST INFRASTRUCTURE ONLY: the checker that the CUDA BDF integrator is compared against
 * (tests/, and the CPU-baseline leg of bench.py).  Nothing in the product links or calls it.
 *
 * The reference integrates time-varying generators with SUNDIALS CVODE, BDF + Newton with the
 * matrix-free SPBCGS Krylov solver, RHS f(t, u) = A(t) u and Jacobian-vector product
 * J v = A(t) v, both through FSPMat::action (tests/test_sundials.cu:67-91, 142, 174-178;
 * problems/hog1p_5species.cu:203-228, 287-336).  SUNDIALS is not vendored and its version is
 * unpinned, so this file restates a published variable-order BDF rather than CVODE's code:
 *
 *   - orders 1..5, quasi-constant step size in backward-difference form (Shampine & Reichelt,
 *     "The MATLAB ODE Suite", SIAM J. Sci. Comput. 18(1), 1997, Sec. 2.3), with the pure BDF
 *     coefficients (kappa = 0): alpha_k = gamma_k = sum_{j<=k} 1/j, local error constant
 *     1/(k+1); step changes by the matrix R(rho) of that paper; order raised or lowered by one
 *     after k+1 equal steps, whichever of k-1, k, k+1 allows the largest step;
 *   - the problem is linear, so the corrector is a single linear solve
 *     (I - c A(t_new)) d = c A(t_new) y_pred - psi,  c = h / alpha_k,
 *     by GMRES (Saad & Schultz 1986) with classical Gram-Schmidt and one re-orthogonalisation
 *     pass, in the weighted inner product <x, y>_w = sum x_i y_i w_i^2 with
 *     w_i = 1 / ((atol + rtol |y_n,i|) sqrt(n)), so that ||.||_w is CVODE's weighted RMS norm;
 *     converged when the residual norm is <= eps_lin; a solve that does not converge within
 *     maxl iterations rejects the step with h halved (CVODE's reaction to a convergence failure);
 *   - local error test err_const_k ||d||_w <= 1; rejected steps shrink h by
 *     max(0.2, 0.9 err^(-1/(k+1)));
 *   - starting step by the algorithm of Hairer, Norsett & Wanner, Solving ODEs I, Sec. II.4;
 *   - output times are hit exactly: the step that would pass t_out is shortened to end on it.
 *
 * The CUDA integrator makes the same decisions from the same formulas; its reductions sum in a
 * different order, so the two agree to rounding except where a decision sits on a threshold.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_OK 0
#define ORC_ERR_ARG 1
#define ORC_ERR_ALLOC 3
#define ORC_ERR_NONFINITE 5
#define ORC_ERR_STEP_LIMIT 6

#define BDF_MAX_ORDER 5
#define BDF_NHIST (BDF_MAX_ORDER + 3)

void orc_spmv(int64_t n, int nr, const int *rowptr, const int *col, const double *val, const double *coefs,
              const double *x, double beta, double *y);

typedef void (*orc_tcoef_fn)(double t, double *c, void *user);

typedef struct {
    double t, h, last_err;
    int order, pad;
    int64_t n_steps, n_reject, n_matvec, n_lin_iters, n_lin_fail;
} orc_bdf_stats;

typedef struct {
    int64_t n;
    int nr;
    const int *rowptr, *col;
    const double *val;
    const double *coefs; /* fixed coefficients, or NULL to call tcoef */
    orc_tcoef_fn tcoef;
    void *user;
    double *cbuf;
    int64_t *n_matvec;
} bdf_op;

/* y = alpha A(t) x (+ y when accumulate) */
static int bdf_apply(const bdf_op *A, double t, double alpha, const double *x, int accumulate, double *y,
                     double *tmp) {
    const double *c = A->coefs;
    if (!c) {
        A->tcoef(t, A->cbuf, A->user);
        for (int r = 0; r < A->nr; ++r)
            if (!isfinite(A->cbuf[r])) return ORC_ERR_NONFINITE;
        c = A->cbuf;
    }
    orc_spmv(A->n, A->nr, A->rowptr, A->col, A->val, c, x, 0.0, tmp);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < A->n; ++i) y[i] = (accumulate ? y[i] : 0.0) + alpha * tmp[i];
    (*A->n_matvec)++;
    return ORC_OK;
}

/* Weighted dot product in a fixed summation order whatever the thread count (64 fixed blocks, then
 * the block sums in order), so that the integrator's decisions do not change from run to run. */
static double wdot(int64_t n, const double *x, const double *y, const double *w) {
    enum { NB = 64 };
    double part[NB];
    if (n < 8192) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) s += x[i] * y[i] * w[i] * w[i];
        return s;
    }
#pragma omp parallel for schedule(static)
    for (int b = 0; b < NB; ++b) {
        const int64_t lo = n * b / NB, hi = n * (b + 1) / NB;
        double s = 0.0;
        for (int64_t i = lo; i < hi; ++i) s += x[i] * y[i] * w[i] * w[i];
        part[b] = s;
    }
    double s = 0.0;
    for (int b = 0; b < NB; ++b) s += part[b];
    return s;
}

static double wnorm(int64_t n, const double *x, const double *w) { return sqrt(wdot(n, x, x, w)); }

static void set_weights(int64_t n, const double *y, double rtol, double atol, double *w) {
    const double sq = sqrt((double)n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) w[i] = 1.0 / ((atol + rtol * fabs(y[i])) * sq);
}

/* R(rho) of Shampine & Reichelt: R[i][j] = prod_{l=1..i} (l - 1 - rho j) / l, R[0][j] = 1, R[i][0] = 0 (i > 0). */
static void bdf_R(int k, double rho, double R[BDF_MAX_ORDER + 1][BDF_MAX_ORDER + 1]) {
    for (int j = 0; j <= k; ++j) R[0][j] = 1.0;
    for (int i = 1; i <= k; ++i) {
        R[i][0] = 0.0;
        for (int j = 1; j <= k; ++j) R[i][j] = R[i - 1][j] * ((i - 1) - rho * j) / (double)i;
    }
}

/* Mixing matrix T of a step-size change by rho at order k: D_i <- sum_j T[i][j] D_j, T = (R(rho) R(1))^T. */
void orc_bdf_change_matrix(int k, double rho, double *T /* (k+1)^2 row-major */) {
    double R[BDF_MAX_ORDER + 1][BDF_MAX_ORDER + 1], U[BDF_MAX_ORDER + 1][BDF_MAX_ORDER + 1];
    bdf_R(k, rho, R);
    bdf_R(k, 1.0, U);
    for (int i = 0; i <= k; ++i)
        for (int j = 0; j <= k; ++j) {
            double s = 0.0; /* (R U)[j][i] */
            for (int l = 0; l <= k; ++l) s += R[j][l] * U[l][i];
            T[i * (k + 1) + j] = s;
        }
}

static void change_D(int64_t n, int k, double rho, double **D, double *tmp) {
    double T[(BDF_MAX_ORDER + 1) * (BDF_MAX_ORDER + 1)];
    orc_bdf_change_matrix(k, rho, T);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double old[BDF_MAX_ORDER + 1];
        for (int j = 0; j <= k; ++j) old[j] = D[j][i];
        for (int r = 0; r <= k; ++r) {
            double s = 0.0;
            for (int j = 0; j <= k; ++j) s += T[r * (k + 1) + j] * old[j];
            D[r][i] = s;
        }
    }
    (void)tmp;
}

/* GMRES on (I - c A(t)) d = b in the w-inner product.  V holds maxl+1 vectors of n.
 * Returns 1 when converged (d written), 0 when not, <0 on error. */
static int bdf_gmres(const bdf_op *A, double t, double c, const double *b, const double *w, int maxl, double eps_lin,
                     double *V, double *d, double *tmp, int64_t *iters) {
    const int64_t n = A->n;
    double H[(64 + 1) * 64], g[65], cs[64], sn[64], y[64];
    memset(H, 0, sizeof(H));
    const double beta = wnorm(n, b, w);
    if (!isfinite(beta)) return -ORC_ERR_NONFINITE;
    if (beta <= eps_lin) {
        memset(d, 0, sizeof(double) * (size_t)n);
        return 1;
    }
    for (int64_t i = 0; i < n; ++i) V[i] = b[i] / beta;
    g[0] = beta;
    int J = 0, conv = 0;
    for (int j = 0; j < maxl; ++j) {
        double *vj = V + (int64_t)j * n, *q = V + (int64_t)(j + 1) * n;
        memcpy(q, vj, sizeof(double) * (size_t)n);
        int rc = bdf_apply(A, t, -c, vj, 1, q, tmp);
        if (rc) return -rc;
        (*iters)++;
        double h1[64], h2[64];
        for (int pass = 0; pass < 2; ++pass) {
            double *hh = pass ? h2 : h1;
            for (int l = 0; l <= j; ++l) hh[l] = wdot(n, V + (int64_t)l * n, q, w);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) {
                double s = q[i];
                for (int l = 0; l <= j; ++l) s -= hh[l] * V[(int64_t)l * n + i];
                q[i] = s;
            }
        }
        const double hn = wnorm(n, q, w);
        if (!isfinite(hn)) return -ORC_ERR_NONFINITE;
        double *col = H + (int64_t)j * 65;
        for (int l = 0; l <= j; ++l) col[l] = h1[l] + h2[l];
        col[j + 1] = hn;
        for (int l = 0; l < j; ++l) { /* earlier rotations */
            const double a = col[l], bb = col[l + 1];
            col[l] = cs[l] * a + sn[l] * bb;
            col[l + 1] = -sn[l] * a + cs[l] * bb;
        }
        const double a = col[j], bb = col[j + 1];
        const double r = hypot(a, bb);
        cs[j] = r > 0.0 ? a / r : 1.0;
        sn[j] = r > 0.0 ? bb / r : 0.0;
        col[j] = r;
        col[j + 1] = 0.0;
        g[j + 1] = -sn[j] * g[j];
        g[j] = cs[j] * g[j];
        J = j + 1;
        if (fabs(g[j + 1]) <= eps_lin || hn == 0.0) {
            conv = 1;
            break;
        }
        if (j + 1 < maxl) {
            const double inv = 1.0 / hn;
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) q[i] *= inv;
        }
    }
    if (!conv) return 0;
    for (int i = J - 1; i >= 0; --i) { /* back substitution R y = g */
        double s = g[i];
        for (int l = i + 1; l < J; ++l) s -= H[(int64_t)l * 65 + i] * y[l];
        y[i] = s / H[(int64_t)i * 65 + i];
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int l = 0; l < J; ++l) s += y[l] * V[(int64_t)l * n + i];
        d[i] = s;
    }
    return 1;
}

/*
 * Integrates dp/dt = A(t) p from t0 through the increasing output times, writing p(times[k]) to
 * out + k n.  A(t) = sum_r c_r(t) A_r with c = coefs (time-invariant) or tcoef(t).
 * h_init <= 0: automatic starting step.  h_max <= 0: unbounded.
 */
int orc_bdf(int64_t n, int nr, const int *rowptr, const int *col, const double *val, const double *coefs,
            orc_tcoef_fn tcoef, void *user, double t0, const double *y0, const double *times, int n_times,
            double *out, double rtol, double atol, int maxl, double eps_lin, double h_init, double h_max,
            int64_t max_steps, orc_bdf_stats *st) {
    if (n < 1 || nr < 1 || nr > 256 || (!coefs && !tcoef) || n_times < 1 || !(rtol > 0.0) || !(atol > 0.0) || maxl < 1 ||
        maxl > 64 || !(eps_lin > 0.0))
        return ORC_ERR_ARG;
    for (int k = 0; k < n_times; ++k)
        if (!(times[k] >= (k ? times[k - 1] : t0))) return ORC_ERR_ARG;
    memset(st, 0, sizeof(*st));
    double cbuf[256];
    bdf_op A = {n, nr, rowptr, col, val, coefs, tcoef, user, cbuf, &st->n_matvec};
    const size_t vb = sizeof(double) * (size_t)n;
    double *store = (double *)malloc(vb * (size_t)(BDF_NHIST + maxl + 1 + 5));
    if (!store) return ORC_ERR_ALLOC;
    double *D[BDF_NHIST];
    for (int j = 0; j < BDF_NHIST; ++j) D[j] = store + (size_t)j * n;
    double *V = store + (size_t)BDF_NHIST * n;
    double *w = V + (size_t)(maxl + 1) * n, *ypred = w + n, *b = ypred + n, *d = b + n, *tmp = d + n;
    memset(store, 0, vb * BDF_NHIST);
    memcpy(D[0], y0, vb);

    double gam[BDF_MAX_ORDER + 2], econst[BDF_MAX_ORDER + 2];
    gam[0] = 0.0;
    for (int k = 1; k <= BDF_MAX_ORDER + 1; ++k) gam[k] = gam[k - 1] + 1.0 / k;
    for (int k = 0; k <= BDF_MAX_ORDER + 1; ++k) econst[k] = 1.0 / (k + 1);
    const double safety = 0.9, min_factor = 0.2, max_factor = 10.0;
    const double hmax = h_max > 0.0 ? h_max : INFINITY;

    double t = t0, h = 0.0, err_last = 0.0;
    int order = 1, n_equal = 0, rc = ORC_OK, started = 0;
    set_weights(n, D[0], rtol, atol, w);

    for (int io = 0; io < n_times && rc == ORC_OK; ++io) {
        const double t_out = times[io];
        if (!started && t_out > t) {
            /* starting step and D[1] = h f(t0, y0) */
            rc = bdf_apply(&A, t, 1.0, D[0], 0, b, tmp); /* b = f0 */
            if (rc) break;
            if (h_init > 0.0) {
                h = h_init;
            } else {
                const double d0 = wnorm(n, D[0], w), d1 = wnorm(n, b, w);
                double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
                h0 = fmin(h0, t_out - t);
                for (int64_t i = 0; i < n; ++i) ypred[i] = D[0][i] + h0 * b[i];
                rc = bdf_apply(&A, t + h0, 1.0, ypred, 0, d, tmp); /* d = f1 */
                if (rc) break;
                for (int64_t i = 0; i < n; ++i) tmp[i] = (d[i] - b[i]) / h0;
                const double d2 = wnorm(n, tmp, w);
                const double h1 = (d1 <= 1e-15 && d2 <= 1e-15) ? fmax(1e-6, h0 * 1e-3) : sqrt(0.01 / fmax(d1, d2));
                h = fmin(100.0 * h0, h1);
            }
            h = fmin(fmin(h, hmax), t_out - t);
            for (int64_t i = 0; i < n; ++i) D[1][i] = h * b[i];
            started = 1;
        }
        while (rc == ORC_OK && t < t_out) {
            if (t_out - t <= 4.0 * 2.220446049250313e-16 * fmax(fabs(t), fabs(t_out))) {
                t = t_out;
                break;
            }
            if (st->n_steps >= max_steps) {
                rc = ORC_ERR_STEP_LIMIT;
                break;
            }
            if (h > hmax) {
                change_D(n, order, hmax / h, D, tmp);
                h = hmax;
                n_equal = 0;
            }
            int landing = 0;
            if (t + h >= t_out) {
                const double rho = (t_out - t) / h;
                if (rho != 1.0) change_D(n, order, rho, D, tmp);
                h = t_out - t;
                n_equal = 0;
                landing = 1;
            }
            if (!(h > 4.0 * 2.220446049250313e-16 * fabs(t))) {
                rc = ORC_ERR_STEP_LIMIT; /* step size underflow */
                break;
            }
            const double t_new = landing ? t_out : t + h;
            const double alpha = gam[order], c = h / alpha;
            /* predictor and psi: ypred = sum_{j<=k} D_j, b = -(sum_{1<=j<=k} gamma_j D_j) / alpha */
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) {
                double yp = 0.0, ps = 0.0;
                for (int j = 0; j <= order; ++j) yp += D[j][i];
                for (int j = 1; j <= order; ++j) ps += gam[j] * D[j][i];
                ypred[i] = yp;
                b[i] = -ps / alpha;
            }
            rc = bdf_apply(&A, t_new, c, ypred, 1, b, tmp);
            if (rc) break;
            int conv = bdf_gmres(&A, t_new, c, b, w, maxl, eps_lin, V, d, tmp, &st->n_lin_iters);
            if (conv < 0) {
                rc = -conv;
                break;
            }
            if (!conv) {
                st->n_lin_fail++;
                change_D(n, order, 0.5, D, tmp);
                h *= 0.5;
                n_equal = 0;
                continue;
            }
            const double err = econst[order] * wnorm(n, d, w);
            if (!isfinite(err)) {
                rc = ORC_ERR_NONFINITE;
                break;
            }
            if (err > 1.0) {
                const double rho = fmax(min_factor, safety * pow(err, -1.0 / (order + 1)));
                change_D(n, order, rho, D, tmp);
                h *= rho;
                n_equal = 0;
                st->n_reject++;
                continue;
            }
            /* accept: D_{k+2} = d - D_{k+1}, D_{k+1} = d, D_j += D_{j+1} for j = k..0 */
            const int k = order;
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) {
                const double di = d[i];
                D[k + 2][i] = di - D[k + 1][i];
                D[k + 1][i] = di;
                for (int j = k; j >= 0; --j) D[j][i] += D[j + 1][i];
            }
            t = t_new;
            st->n_steps++;
            n_equal++;
            err_last = err;
            set_weights(n, D[0], rtol, atol, w);
            if (n_equal >= order + 1) {
                const double em = order > 1 ? econst[order - 1] * wnorm(n, D[order], w) : INFINITY;
                const double ep = order < BDF_MAX_ORDER ? econst[order + 1] * wnorm(n, D[order + 2], w) : INFINITY;
                const double fm = pow(em, -1.0 / order), f0 = pow(err, -1.0 / (order + 1)),
                             fp = pow(ep, -1.0 / (order + 2));
                int delta = 0;
                double best = f0;
                if (fm > best) { best = fm; delta = -1; }
                if (fp > best) { best = fp; delta = 1; }
                order += delta;
                const double rho = fmin(max_factor, safety * best);
                change_D(n, order, rho, D, tmp);
                h *= rho;
                n_equal = 0;
            }
        }
        if (rc == ORC_OK) memcpy(out + (size_t)io * n, D[0], vb);
    }
    st->t = t;
    st->h = h;
    st->order = order;
    st->last_err = err_last;
    free(store);
    return rc;
}
