/*
 * fsp_oracle.c -- FP64 host oracle for the Finite State Projection generator path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product path is
 * compared against (by tests/, by __graft_entry__.smoke(), and as the timed CPU baseline
 * in bench.py).  Nothing in the product (cuda_fsp_b200/, include/) may link or call it.
 *
 * It restates, in plain C with OpenMP, the algorithms of voduchuy/CUDA_FSP:
 *   - state indexing          src/cme_util.cu:5-22, 24-41, 43-53, 55-62
 *   - per-reaction CSR build  src/fspmat_csr_kernels.cu:7-51 (nnz per row), 53-94 (fill),
 *                             138-248 (driver: enumerate -> count -> scan -> fill)
 *   - generator action        src/fspmat_csr_kernels.cu:123-136 (y += c_r A_r x, r = 0..nr-1)
 *   - Kronecker factor tables src/fspmat_kron_kernels.cu:170-190
 *   - Krylov exp(tA)v         src/KryExpvFSP.cu:38-188 (Expokit-style step control)
 *   - dense exp(tau*H)        the reference calls Armadillo expmat (src/KryExpvFSP.cu:125,
 *                             version unpinned); restated here as the published
 *                             scaling-and-squaring Pade(13,13) method (Higham, SIAM J. Matrix
 *                             Anal. Appl. 26(4), 2005), coefficients computed from the Pade
 *                             formula c_j = (2m-j)! m! / ((2m)! j! (m-j)!).
 *
 * Deviations from the reference, all deliberate (the reference's own defects):
 *   - KryExpvFSP::k1 is reset to 2 at the start of every step (reference keeps it at 0 after
 *     the first happy breakdown and then skips every later error estimate, KryExpvFSP.h:61).
 *   - pi is M_PI, not 3.1416 (KryExpvFSP.cu:48).
 *   - a zero start vector returns immediately (the reference divides by beta = 0).
 *   - a non-finite beta / error estimate is reported as an error instead of looping.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_ERR_ARG 1
#define ORC_ERR_ALLOC 3
#define ORC_ERR_NONFINITE 5
#define ORC_ERR_STEP_LIMIT 6

/* ------------------------------------------------------------------------------------------
 * State indexing: mixed radix, species 0 varies fastest.  src/cme_util.cu:5-22, 55-62
 * ---------------------------------------------------------------------------------------- */
int64_t orc_num_states(int ns, const int *bounds) {
    int64_t n = 1;
    for (int s = 0; s < ns; ++s) n *= (int64_t)bounds[s] + 1;
    return n;
}

void orc_indx2state(int64_t indx, int *state, int ns, const int *bounds) {
    for (int s = 0; s < ns; ++s) {
        state[s] = (int)(indx % ((int64_t)bounds[s] + 1));
        indx /= ((int64_t)bounds[s] + 1);
    }
}

int64_t orc_state2indx(const int *state, int ns, const int *bounds) {
    int64_t indx = 0, nprod = 1;
    for (int s = 0; s < ns; ++s) {
        indx += (int64_t)state[s] * nprod;
        nprod *= (int64_t)bounds[s] + 1;
    }
    return indx;
}

/* AoS state table, state i at states[i*ns .. i*ns+ns-1].  src/cme_util.cu:24-41 */
void orc_get_states(int ns, const int *bounds, int *states) {
    int64_t n = orc_num_states(ns, bounds);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) orc_indx2state(i, states + i * ns, ns, bounds);
}

/* x +/- nu_r using the CSR stoichiometry (rows = reactions).  src/cme_util.cu:43-53 */
static void orc_reachable_state(const int *state, int *rstate, int reaction, int direction, int ns,
                                const int *sv, const int *sc, const int *sr) {
    for (int k = 0; k < ns; ++k) rstate[k] = state[k];
    for (int i = sr[reaction]; i < sr[reaction + 1]; ++i) rstate[sc[i]] += direction * sv[i];
}

/* ------------------------------------------------------------------------------------------
 * Propensity sources.
 *   kind 0: factor tables, a_r(x) = prod_s f_{r,s}(x_s); layout of the reference's
 *           SDKronMatSet::vals: reaction-major, then species, then x_s = 0..b_s
 *           (src/fspmat_kron_kernels.cu:170-190).  The product is taken as
 *           ((1 * f_{r,0}) * f_{r,1}) * ... in species order.
 *   kind 1: the toggle-switch model of the reference tests (tests/test_fsp_mat.cu:19-50):
 *           2 species, 6 reactions, Hill repression.
 *   kind 2: a non-factorisable test model: the toggle switch with reaction 1 replaced by
 *           1 / (1 + ayx*x1^nyx + 0.05*x0) and reaction 4 by x0*x1/(10 + x0 + x1) + 1.
 * ---------------------------------------------------------------------------------------- */
typedef struct {
    int kind;
    int ns;
    const int *bounds;
    const double *tables; /* kind 0 */
} orc_prop;

static const double T_ayx = 2.6e-3, T_axy = 6.1e-3, T_nyx = 3e0, T_nxy = 2.1e0;

static double orc_toggle(const int *x, int r) {
    switch (r) {
        case 0: return 1.0;
        case 1: return 1.0 / (1.0 + T_ayx * pow(1.0 * x[1], T_nyx));
        case 2: return 1.0 * x[0];
        case 3: return 1.0;
        case 4: return 1.0 / (1.0 + T_axy * pow(1.0 * x[0], T_nxy));
        case 5: return 1.0 * x[1];
        default: return 0.0;
    }
}

static double orc_nonfact(const int *x, int r) {
    switch (r) {
        case 1: return 1.0 / (1.0 + T_ayx * pow(1.0 * x[1], T_nyx) + 0.05 * x[0]);
        case 4: return (1.0 * x[0]) * (1.0 * x[1]) / (10.0 + x[0] + x[1]) + 1.0;
        default: return orc_toggle(x, r);
    }
}

static double orc_eval_prop(const orc_prop *p, const int *x, int r) {
    if (p->kind == 0) {
        int64_t stride = 0;
        for (int s = 0; s < p->ns; ++s) stride += p->bounds[s] + 1;
        const double *t = p->tables + (int64_t)r * stride;
        double a = 1.0;
        for (int s = 0; s < p->ns; ++s) {
            a *= t[x[s]];
            t += p->bounds[s] + 1;
        }
        return a;
    }
    if (p->kind == 1) return orc_toggle(x, r);
    return orc_nonfact(x, r);
}

/* Propensity value a_r(x) for a state given by its multi-index (used by tests). */
double orc_propensity(int kind, int ns, const int *bounds, const double *tables, const int *x, int r) {
    orc_prop p = {kind, ns, bounds, tables};
    return orc_eval_prop(&p, x, r);
}

/* Factor tables from the toggle model's factorised form (tests/test_fsp_mat.cu:52-84),
 * filled in the reference's order (src/fspmat_kron_kernels.cu:170-190). */
static double orc_toggle_factor(int x, int s, int r) {
    double v = 1.0;
    switch (r) {
        case 1: if (s == 1) v = 1.0 / (1.0 + T_ayx * pow(1.0 * x, T_nyx)); break;
        case 2: if (s == 0) v = 1.0 * x; break;
        case 4: if (s == 0) v = 1.0 / (1.0 + T_axy * pow(1.0 * x, T_nxy)); break;
        case 5: if (s == 1) v = 1.0 * x; break;
        default: break;
    }
    return v;
}

void orc_toggle_factor_tables(const int *bounds, double *vals) {
    int iv = 0;
    for (int r = 0; r < 6; ++r)
        for (int s = 0; s < 2; ++s)
            for (int x = 0; x <= bounds[s]; ++x) vals[iv++] = orc_toggle_factor(x, s, r);
}

/* ------------------------------------------------------------------------------------------
 * Per-reaction CSR assembly.  src/fspmat_csr_kernels.cu:7-94, 138-248.
 * Row i of A_r holds -a_r(x_i) on the diagonal and a_r(x_i - nu_r) at column idx(x_i - nu_r)
 * when x_i - nu_r lies inside the box, columns in increasing order.
 * Output arrays (caller-allocated, nr blocks): rowptr[nr*(n+1)], col[nr*2n], val[nr*2n],
 * nnz[nr].  Block r starts at rowptr + r*(n+1) and col/val + r*2n.
 * ---------------------------------------------------------------------------------------- */
int orc_assemble_csr(int ns, int nr, const int *bounds, const int *sv, const int *sc, const int *sr,
                     int prop_kind, const double *tables, int *rowptr, int *col, double *val,
                     int64_t *nnz_out) {
    int64_t n = orc_num_states(ns, bounds);
    orc_prop p = {prop_kind, ns, bounds, tables};
    int *states = (int *)malloc(sizeof(int) * (size_t)(n * ns));
    int *off = (int *)malloc(sizeof(int) * (size_t)n);
    if (!states || !off) { free(states); free(off); return ORC_ERR_ALLOC; }
    orc_get_states(ns, bounds, states);
    for (int r = 0; r < nr; ++r) {
        int *rp = rowptr + (int64_t)r * (n + 1);
        int *cl = col + (int64_t)r * 2 * n;
        double *vl = val + (int64_t)r * 2 * n;
        /* nnz per row and off-diagonal column (fspmat_csr_get_nnz_per_row, :7-51) */
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            int rs[64];
            orc_reachable_state(states + i * ns, rs, r, -1, ns, sv, sc, sr);
            int reachable = 1;
            for (int k = 0; k < ns; ++k) reachable = reachable && rs[k] >= 0 && rs[k] <= bounds[k];
            rp[i + 1] = 1 + reachable;
            off[i] = reachable ? (int)orc_state2indx(rs, ns, bounds) : -1;
        }
        /* inclusive scan (thrust::inclusive_scan, :209-210) */
        rp[0] = 0;
        for (int64_t i = 0; i < n; ++i) rp[i + 1] += rp[i];
        nnz_out[r] = rp[n];
        /* fill (fspmat_csr_fill_data, :53-94) */
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            int o = off[i], base = rp[i];
            double d = -orc_eval_prop(&p, states + i * ns, r);
            if (o >= 0) {
                double a = orc_eval_prop(&p, states + (int64_t)o * ns, r);
                int idiag = (o > i) ? base : base + 1, ioff = (o > i) ? base + 1 : base;
                vl[idiag] = d; cl[idiag] = (int)i;
                vl[ioff] = a; cl[ioff] = o;
            } else {
                vl[base] = d; cl[base] = (int)i;
            }
        }
    }
    free(states);
    free(off);
    return ORC_OK;
}

/* y = beta*y + sum_r c_r A_r x, reactions applied in order r = 0..nr-1 as the reference's
 * nr csrmv calls do (src/fspmat_csr_kernels.cu:123-136). */
void orc_spmv(int64_t n, int nr, const int *rowptr, const int *col, const double *val,
              const double *coefs, const double *x, double beta, double *y) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double acc = (beta == 0.0) ? 0.0 : beta * y[i];
        for (int r = 0; r < nr; ++r) {
            const int *rp = rowptr + (int64_t)r * (n + 1);
            const int *cl = col + (int64_t)r * 2 * n;
            const double *vl = val + (int64_t)r * 2 * n;
            double s = 0.0;
            for (int k = rp[i]; k < rp[i + 1]; ++k) s += vl[k] * x[cl[k]];
            acc += coefs[r] * s;
        }
        y[i] = acc;
    }
}

/* Elementwise scale for tolerances: z = sum_r |c_r| |A_r| |x|. */
void orc_abs_spmv(int64_t n, int nr, const int *rowptr, const int *col, const double *val,
                  const double *coefs, const double *x, double *z) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double acc = 0.0;
        for (int r = 0; r < nr; ++r) {
            const int *rp = rowptr + (int64_t)r * (n + 1);
            const int *cl = col + (int64_t)r * 2 * n;
            const double *vl = val + (int64_t)r * 2 * n;
            for (int k = rp[i]; k < rp[i + 1]; ++k) acc += fabs(coefs[r]) * fabs(vl[k]) * fabs(x[cl[k]]);
        }
        z[i] = acc;
    }
}

/* ||A||_1 = max column sum of |sum_r c_r A_r| (used as anorm by callers that want it). */
double orc_norm1(int64_t n, int nr, const int *rowptr, const int *col, const double *val,
                 const double *coefs) {
    double *cs = (double *)calloc((size_t)n, sizeof(double));
    for (int64_t i = 0; i < n; ++i)
        for (int r = 0; r < nr; ++r) {
            const int *rp = rowptr + (int64_t)r * (n + 1);
            const int *cl = col + (int64_t)r * 2 * n;
            const double *vl = val + (int64_t)r * 2 * n;
            for (int k = rp[i]; k < rp[i + 1]; ++k) cs[cl[k]] += fabs(coefs[r] * vl[k]);
        }
    double m = 0.0;
    for (int64_t i = 0; i < n; ++i) m = cs[i] > m ? cs[i] : m;
    free(cs);
    return m;
}

/* ------------------------------------------------------------------------------------------
 * Dense exp by scaling and squaring with the diagonal Pade(13,13) approximant.
 * A and F are column-major k x k.  Higham 2005: theta_13 = 5.371920351148152.
 * ---------------------------------------------------------------------------------------- */
static void orc_gemm(int k, const double *A, const double *B, double *C) {
    for (int j = 0; j < k; ++j)
        for (int i = 0; i < k; ++i) {
            double s = 0.0;
            for (int l = 0; l < k; ++l) s += A[i + l * k] * B[l + j * k];
            C[i + j * k] = s;
        }
}

int orc_expm(int k, const double *A_in, double *F) {
    const int m = 13;
    double c[14];
    c[0] = 1.0;
    for (int j = 0; j < m; ++j) c[j + 1] = c[j] * (double)(m - j) / ((double)(j + 1) * (double)(2 * m - j));
    size_t sz = (size_t)k * k;
    double *W = (double *)malloc(sizeof(double) * sz * 9);
    if (!W) return ORC_ERR_ALLOC;
    double *A = W, *A2 = W + sz, *A4 = W + 2 * sz, *A6 = W + 3 * sz, *U = W + 4 * sz, *V = W + 5 * sz,
           *T = W + 6 * sz, *P = W + 7 * sz, *Q = W + 8 * sz;
    double nrm = 0.0;
    for (int j = 0; j < k; ++j) {
        double cs = 0.0;
        for (int i = 0; i < k; ++i) cs += fabs(A_in[i + j * k]);
        nrm = cs > nrm ? cs : nrm;
    }
    if (!isfinite(nrm)) { free(W); return ORC_ERR_NONFINITE; }
    int s = 0;
    if (nrm > 5.371920351148152) s = (int)ceil(log2(nrm / 5.371920351148152));
    double scale = ldexp(1.0, -s);
    for (size_t i = 0; i < sz; ++i) A[i] = A_in[i] * scale;
    orc_gemm(k, A, A, A2);
    orc_gemm(k, A2, A2, A4);
    orc_gemm(k, A4, A2, A6);
    /* U = A (A6 (c13 A6 + c11 A4 + c9 A2) + c7 A6 + c5 A4 + c3 A2 + c1 I) */
    for (size_t i = 0; i < sz; ++i) T[i] = c[13] * A6[i] + c[11] * A4[i] + c[9] * A2[i];
    orc_gemm(k, A6, T, P);
    for (size_t i = 0; i < sz; ++i) P[i] += c[7] * A6[i] + c[5] * A4[i] + c[3] * A2[i];
    for (int i = 0; i < k; ++i) P[i + i * k] += c[1];
    orc_gemm(k, A, P, U);
    /* V = A6 (c12 A6 + c10 A4 + c8 A2) + c6 A6 + c4 A4 + c2 A2 + c0 I */
    for (size_t i = 0; i < sz; ++i) T[i] = c[12] * A6[i] + c[10] * A4[i] + c[8] * A2[i];
    orc_gemm(k, A6, T, V);
    for (size_t i = 0; i < sz; ++i) V[i] += c[6] * A6[i] + c[4] * A4[i] + c[2] * A2[i];
    for (int i = 0; i < k; ++i) V[i + i * k] += c[0];
    /* solve (V - U) F = (V + U) by Gaussian elimination with partial pivoting */
    for (size_t i = 0; i < sz; ++i) { P[i] = V[i] - U[i]; Q[i] = V[i] + U[i]; }
    for (int col = 0; col < k; ++col) {
        int piv = col;
        for (int i = col + 1; i < k; ++i)
            if (fabs(P[i + col * k]) > fabs(P[piv + col * k])) piv = i;
        if (piv != col) {
            for (int j = 0; j < k; ++j) {
                double t = P[col + j * k]; P[col + j * k] = P[piv + j * k]; P[piv + j * k] = t;
                t = Q[col + j * k]; Q[col + j * k] = Q[piv + j * k]; Q[piv + j * k] = t;
            }
        }
        double d = P[col + col * k];
        for (int i = col + 1; i < k; ++i) {
            double f = P[i + col * k] / d;
            if (f == 0.0) continue;
            for (int j = col; j < k; ++j) P[i + j * k] -= f * P[col + j * k];
            for (int j = 0; j < k; ++j) Q[i + j * k] -= f * Q[col + j * k];
        }
    }
    for (int j = 0; j < k; ++j)
        for (int i = k - 1; i >= 0; --i) {
            double sum = Q[i + j * k];
            for (int l = i + 1; l < k; ++l) sum -= P[i + l * k] * F[l + j * k];
            F[i + j * k] = sum / P[i + i * k];
        }
    for (int q = 0; q < s; ++q) {
        orc_gemm(k, F, F, T);
        memcpy(F, T, sizeof(double) * sz);
    }
    free(W);
    return ORC_OK;
}

/* ------------------------------------------------------------------------------------------
 * Krylov exp(t_final * A) v, restating KryExpvFSP::step/solve (src/KryExpvFSP.cu:38-188):
 * Expokit step-size control (delta = 1.2, gamma = 0.9), classical Gram-Schmidt Arnoldi
 * (two gemv passes, :70-109) with optional incomplete orthogonalisation against the last
 * q_iop vectors, the augmented (m+2)x(m+2) Hessenberg matrix, the phi1/phi2 local error
 * estimate (:122-158), and 2-significant-digit step rounding (:153-154, :172-174).
 * ---------------------------------------------------------------------------------------- */
typedef struct {
    int64_t n;
    int nr;
    const int *rowptr, *col;
    const double *val, *coefs;
} orc_op;

static void orc_op_apply(const orc_op *A, const double *x, double *y) {
    orc_spmv(A->n, A->nr, A->rowptr, A->col, A->val, A->coefs, x, 0.0, y);
}

/* x . y in a fixed summation order whatever the thread count: 64 fixed blocks summed in parallel,
 * then the block sums in order (an OpenMP reduction combines per-thread sums in an unspecified
 * order, which made borderline breakdown decisions change from run to run). */
static double orc_dot(int64_t n, const double *x, const double *y) {
    enum { NB = 64 };
    double part[NB];
    if (n < 8192) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) s += x[i] * y[i];
        return s;
    }
#pragma omp parallel for schedule(static)
    for (int b = 0; b < NB; ++b) {
        const int64_t lo = n * b / NB, hi = n * (b + 1) / NB;
        double s = 0.0;
        for (int64_t i = lo; i < hi; ++i) s += x[i] * y[i];
        part[b] = s;
    }
    double s = 0.0;
    for (int b = 0; b < NB; ++b) s += part[b];
    return s;
}

static double orc_nrm2(int64_t n, const double *x) { return sqrt(orc_dot(n, x, x)); }

typedef struct {
    int64_t n_steps, n_reject, n_matvec;
    double t_now, last_err;
    int64_t n_breakdown;
} orc_expv_stats;

static double orc_round2(double t) {
    double s = pow(10.0, floor(log10(t)) - 1.0);
    return ceil(t / s) * s;
}

int orc_expv(int64_t n, int nr, const int *rowptr, const int *col, const double *val, const double *coefs,
             double t_final, double *v, int m, double tol, int iop, int q_iop, double anorm,
             int64_t max_nstep, int64_t max_reject, orc_expv_stats *st) {
    if (m < 1 || n < 1 || tol <= 0.0 || anorm <= 0.0) return ORC_ERR_ARG;
    orc_op A = {n, nr, rowptr, col, val, coefs};
    const double delta = 1.2, gamma = 0.9;
    int mp2 = m + 2;
    double *Vb = (double *)malloc(sizeof(double) * (size_t)n * (size_t)mp2);
    double *H = (double *)malloc(sizeof(double) * (size_t)mp2 * mp2);
    double *F = (double *)malloc(sizeof(double) * (size_t)mp2 * mp2);
    double *tH = (double *)malloc(sizeof(double) * (size_t)mp2 * mp2);
    double *h = (double *)malloc(sizeof(double) * (size_t)mp2);
    if (!Vb || !H || !F || !tH || !h) { free(Vb); free(H); free(F); free(tH); free(h); return ORC_ERR_ALLOC; }
    memset(st, 0, sizeof(*st));
    double t_now = 0.0, t_new = 0.0, btol = 0.0, xm = 1.0 / m, err_loc = 0.0;
    int rc = ORC_OK;
    int64_t i_step = 0;
    while (t_now < t_final) {
        if (i_step >= max_nstep) { rc = ORC_ERR_STEP_LIMIT; break; }
        double beta = orc_nrm2(n, v);
        if (!isfinite(beta)) { rc = ORC_ERR_NONFINITE; break; }
        if (beta == 0.0) { t_now = t_final; break; }
        if (i_step == 0) {
            xm = 1.0 / (double)m;
            double fact = pow((m + 1) / exp(1.0), m + 1) * sqrt(2.0 * M_PI * (m + 1));
            t_new = (1.0 / anorm) * pow((fact * tol) / (4.0 * beta * anorm), xm);
            btol = anorm * tol;
        }
        int mb = m, k1 = 2;
        double tau = fmin(t_final - t_now, t_new);
        memset(H, 0, sizeof(double) * (size_t)mp2 * mp2);
        for (int64_t i = 0; i < n; ++i) Vb[i] = v[i] / beta;
        int istart = 0;
        for (int j = 0; j < m; ++j) {
            double *w = Vb + (int64_t)(j + 1) * n;
            orc_op_apply(&A, Vb + (int64_t)j * n, w);
            st->n_matvec++;
            if (iop) istart = (j >= q_iop - 1) ? j - q_iop + 1 : 0;
            /* h = V[istart..j]^T w (first gemv), then w -= V h (second gemv) */
            for (int k = istart; k <= j; ++k) {
                const double *vk = Vb + (int64_t)k * n;
                const double s = orc_dot(n, vk, w);
                h[k] = s;
                H[k + j * mp2] = s;
            }
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) {
                double acc = w[i];
                for (int k = istart; k <= j; ++k) acc -= Vb[(int64_t)k * n + i] * h[k];
                w[i] = acc;
            }
            double s = orc_nrm2(n, w);
            /* The reference's happy-breakdown test (KryExpvFSP.cu:90-98) with the threshold divided by
             * the remaining time when above 1: the jump to t_final that follows then stays within tol
             * (the reference's threshold allows an error of tol per unit of remaining time). */
            if (s < btol / fmax(1.0, t_final - t_now)) {
                k1 = 0;
                mb = j + 1;
                tau = t_final - t_now;
                st->n_breakdown++;
                break;
            }
            H[(j + 1) + j * mp2] = s;
            double sinv = 1.0 / s;
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) w[i] *= sinv;
        }
        double avnorm = 0.0;
        if (k1 != 0) {
            H[(m + 1) + m * mp2] = 1.0;
            orc_op_apply(&A, Vb + (int64_t)mb * n, Vb + (int64_t)(mb + 1) * n);
            st->n_matvec++;
            avnorm = orc_nrm2(n, Vb + (int64_t)(mb + 1) * n);
        }
        int64_t ireject = 0;
        int accepted = 0;
        while (ireject < max_reject) {
            int mx = mb + k1;
            for (int i = 0; i < mp2 * mp2; ++i) tH[i] = tau * H[i];
            if (orc_expm(mp2, tH, F) != ORC_OK) { rc = ORC_ERR_NONFINITE; break; }
            if (k1 == 0) { err_loc = btol; accepted = 1; break; }
            double phi1 = fabs(beta * F[(mx - 2)]), phi2 = fabs(beta * F[(mx - 1)] * avnorm);
            if (phi1 > phi2 * 10.0) { err_loc = phi2; xm = 1.0 / (double)mx; }
            else if (phi1 > phi2) { err_loc = (phi1 * phi2) / (phi1 - phi2); xm = 1.0 / (double)mx; }
            else { err_loc = phi1; xm = 1.0 / (double)(mx - 1); }
            if (!isfinite(err_loc)) { rc = ORC_ERR_NONFINITE; break; }
            if (err_loc <= delta * tau * tol) { accepted = 1; break; }
            tau = gamma * tau * pow(tau * tol / err_loc, xm);
            tau = orc_round2(tau);
            ireject++;
            st->n_reject++;
        }
        if (rc != ORC_OK) break;
        if (!accepted) { rc = ORC_ERR_STEP_LIMIT; break; }
        int mx = mb + (k1 - 1 > 0 ? k1 - 1 : 0);
        /* v = beta * V[:, 0:mx] F(0:mx, 0) */
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int k = 0; k < mx; ++k) acc += Vb[(int64_t)k * n + i] * F[k];
            v[i] = beta * acc;
        }
        /* the step that reaches t_final lands on it exactly (no sub-ulp trailing step) */
        t_now = (tau >= t_final - t_now) ? t_final : t_now + tau;
        if (err_loc > 0.0) {
            t_new = gamma * tau * pow(tau * tol / err_loc, xm);
            t_new = orc_round2(t_new);
        }
        if (!(t_new > 0.0) || !isfinite(t_new)) t_new = t_final - t_now;
        i_step++;
        st->last_err = err_loc;
    }
    st->n_steps = i_step;
    st->t_now = t_now;
    free(Vb); free(H); free(F); free(tH); free(h);
    return rc;
}

/* Number of OpenMP threads the oracle uses. */
int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
