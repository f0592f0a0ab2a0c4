/*
 * cufsp.h -- C ABI of the B200-native Finite State Projection (FSP) engine.
 *
 * Every entry point returns a cufsp_status and never exits the process.  Device pointers are
 * plain `double*` / `int*` in device memory; host pointers are stated as such.  Work is
 * ordered on the `stream` argument (0 = the legacy default stream) and no call synchronises
 * unless its comment says so.  Handles are not thread-safe: use one handle per host thread.
 *
 * Generator convention (shared by all formats):
 *   (A p)(x) = sum_r c_r(t) [ a_r(x - nu_r) p(x - nu_r) 1{x - nu_r in box} - a_r(x) p(x) ]
 * States are the hyper-rectangle 0 <= x_s <= b_s, indexed mixed-radix with species 0 fastest.
 * The diagonal keeps the full outflow even where x + nu_r leaves the box, so 1 - sum(p) is the
 * FSP truncation error.
 */
#ifndef CUFSP_H
#define CUFSP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *cufsp_stream_t; /* == cudaStream_t */

typedef enum {
    CUFSP_SUCCESS = 0,
    CUFSP_ERR_INVALID_ARG = 1,  /* bad argument (null pointer, negative bound, ...) */
    CUFSP_ERR_OVERFLOW = 2,     /* state count does not fit in int32 (the reference's index type) */
    CUFSP_ERR_ALLOC = 3,        /* device or pinned allocation failed */
    CUFSP_ERR_CUDA = 4,         /* a CUDA runtime call failed; see cufsp_last_error() */
    CUFSP_ERR_NONFINITE = 5,    /* NaN/Inf met in coefficients, tables or the Krylov iteration */
    CUFSP_ERR_STEP_LIMIT = 6,   /* Krylov max_nstep / max_reject exhausted */
    CUFSP_ERR_UNSUPPORTED = 7,  /* valid request this build does not implement (e.g. > 32 reactions on KRONECKER) */
    CUFSP_ERR_NO_DEVICE = 8     /* no CUDA device / kernels not loadable */
} cufsp_status;

/* Matrix formats, numbered as the reference's cuFSP::MatrixFormat (src/FSPMat.h:17-19).
 * CSR and HYB are both served by the reaction-major propensity-table format (sparse variant);
 * KRONECKER is the matrix-free factorised kernel. */
typedef enum { CUFSP_FORMAT_CSR = 0, CUFSP_FORMAT_HYB = 1, CUFSP_FORMAT_KRONECKER = 2 } cufsp_format;

/* Device propensity a_r(x): replaces cuFSP::PropFun (src/cme_util.h:25).  Must be a __device__
 * function address taken (cudaMemcpyFromSymbol) in the SAME device-linked module as this
 * library's kernels, i.e. a program linked against libcufsp_static.a with -rdc. */
typedef double (*cufsp_prop_fn)(int *x, int reaction);
/* Host propensity factor f_{r,s}(x_s): replaces cuFSP::PropFactorFun (src/fspmat_kron_kernels.h:13). */
typedef double (*cufsp_prop_factor_fn)(int x, int species, int reaction);
/* Host time coefficients c_r(t) -> out[n_reactions]: replaces cuFSP::TcoefFun (src/FSPMat.h:16),
 * with a user pointer added so C callers can carry state. */
typedef void (*cufsp_tcoef_fn)(double t, double *out, void *user);

/* Model description (all pointers host memory; copied at create).
 * Stoichiometry: CSR with one row per reaction and one column per species (the reference's
 * CSRMatInt stoich argument, src/FSPMat.h:44-50).
 * Propensity source, first non-null wins:
 *   factor_tables : n_reactions * sum_s (b_s + 1) doubles, reaction-major then species then
 *                   x_s = 0..b_s (the layout of SDKronMatSet::vals, src/fspmat_kron_kernels.cu:170-190)
 *   prop_factor   : host factor function, evaluated into such tables at create
 *   prop_device   : device propensity (sparse formats only)
 * tcoef: c_r(t) callback used by cufsp_mat_action; NULL means c_r = 1. */
typedef struct {
    int n_species;
    int n_reactions;
    const int *fsp_bounds;
    const int *stoich_vals;
    const int *stoich_colidxs;
    const int *stoich_rowptrs;
    const double *factor_tables;
    cufsp_prop_factor_fn prop_factor;
    cufsp_prop_fn prop_device;
    cufsp_tcoef_fn tcoef;
    void *tcoef_user;
} cufsp_model_desc;

typedef struct cufsp_mat_s cufsp_mat;
typedef struct cufsp_expv_s cufsp_expv;

/* ---- status ---------------------------------------------------------------------------- */
const char *cufsp_status_string(cufsp_status s);
/* Detail of the last failure on this host thread ("" if none). */
const char *cufsp_last_error(void);

/* ---- state indexing (host) ----------------------------------------------------------------
 * rect_fsp_num_states / indx2state / state2indx, src/cme_util.cu:5-22,55-62 */
cufsp_status cufsp_num_states(int n_species, const int *fsp_bounds, int64_t *n_states);
cufsp_status cufsp_indx2state(int64_t indx, int *state, int n_species, const int *fsp_bounds);
cufsp_status cufsp_state2indx(const int *state, int n_species, const int *fsp_bounds, int64_t *indx);

/* ---- state enumeration (device) -----------------------------------------------------------
 * fsp_get_states, src/cme_util.cu:24-41: d_states[i*n_species + s] = x_s of state i (AoS int32).
 * fsp_bounds is host memory. */
cufsp_status cufsp_get_states(int n_species, const int *fsp_bounds, int *d_states, cufsp_stream_t stream);

/* ---- generator ----------------------------------------------------------------------------
 * cufsp_mat_create replaces both cuFSP::FSPMat constructors (src/FSPMat.cu:10-45 with PropFun,
 * src/FSPMat.cu:49-76 with PropFactorFun).  Synchronises the device once (assembly). */
cufsp_status cufsp_mat_create(const cufsp_model_desc *desc, cufsp_format format, cufsp_mat **out);
cufsp_status cufsp_mat_destroy(cufsp_mat *A);
/* CSR/HYB generator from propensities evaluated by the caller on the host: prop_table[r * n + i] =
 * a_r(x_i) (host, n_reactions * n_states doubles, copied).  For models whose propensity is host code
 * -- the legacy cme::Model::propensity (src/Model.h:14-26), a host function of the state -- rather than
 * a device PropFun or factor tables.  The descriptor's propensity fields are ignored.  Synchronises. */
cufsp_status cufsp_mat_create_table(const cufsp_model_desc *desc, cufsp_format format, const double *prop_table,
                                    cufsp_mat **out);
/* get_n_rows / get_n_species / get_n_reactions, src/FSPMat.cu:108-118 */
cufsp_status cufsp_mat_num_states(const cufsp_mat *A, int64_t *n_states);
cufsp_status cufsp_mat_dims(const cufsp_mat *A, int *n_species, int *n_reactions, cufsp_format *format);

/* FSPMat::action(t, x, y), src/FSPMat.cu:102-105: y += A(t) x with c_r = tcoef(t).
 * x, y: device, n_states doubles, must not overlap. */
cufsp_status cufsp_mat_action(cufsp_mat *A, double t, const double *x, double *y, cufsp_stream_t stream);

/* General form: y = alpha * (sum_r coefs[r] A_r) x + beta * y, beta in {0, 1}.
 * coefs: host, n_reactions doubles (NULL: use tcoef(t)).  Used by the Krylov and BDF drivers. */
cufsp_status cufsp_mat_apply(cufsp_mat *A, double t, const double *coefs, double alpha, const double *x,
                             double beta, double *y, cufsp_stream_t stream);

/* y = alpha A(t)^T x (overwrite), the operator of the adjoint solves; KRONECKER generators only
 * (no counterpart in the reference, whose solvers never apply A^T).  coefs as in cufsp_mat_apply;
 * x and y must not alias.  Asynchronous on `stream`. */
cufsp_status cufsp_mat_apply_transpose(cufsp_mat *A, double t, const double *coefs, double alpha, const double *x,
                                       double *y, cufsp_stream_t stream);

/* FSPMat::action with HOST buffers: y_host += A(t) x_host.  Copies in, computes and copies out in
 * a pipeline of slabs on internal streams; returns after y_host is written (synchronous).
 * x_host / y_host should be pinned (cudaHostAlloc) for full PCIe bandwidth. */
cufsp_status cufsp_mat_action_host(cufsp_mat *A, double t, const double *x_host, double *y_host);

/* Watchdog of the TMA-fed KRONECKER kernel: *tripped = 1 when one of its bounded shared-memory
 * barrier waits expired since the previous call (the affected output is then incomplete); the flag
 * is reset.  Synchronises the device.  The drivers that synchronise anyway -- Krylov steps, BDF steps,
 * the FSP solvers, the gradient and cufsp_mat_action_host -- read the same flag after every step and
 * return CUFSP_ERR_CUDA when it is set; a caller of the asynchronous cufsp_mat_action/apply checks it
 * here. */
cufsp_status cufsp_mat_watchdog(cufsp_mat *A, int *tripped);

/* Which kernel serves this generator's action, as text (e.g. the runtime-specialised plane kernel of
 * a KRONECKER generator, or the general one with the reason the plane kernel was not used).
 * Writes at most len bytes including the terminating NUL.  No counterpart in the reference. */
cufsp_status cufsp_mat_describe(const cufsp_mat *A, char *buf, size_t len);

/* Sparse-format export for checking (HYB/CSR formats only): props[r*n + i] = a_r(x_i). */
cufsp_status cufsp_mat_export_propensities(const cufsp_mat *A, double *d_props, cufsp_stream_t stream);

/* ---- Krylov exp(tA)v -------------------------------------------------------------------------
 * Replaces cuFSP::KryExpvFSP (src/KryExpvFSP.h:20-108, src/KryExpvFSP.cu:6-203).
 * The Arnoldi basis, the Hessenberg matrix and all reductions stay on the device; one
 * device->host read of the (m+2)^2 Hessenberg matrix per step drives the host step control. */
typedef struct {
    int64_t n_steps;     /* accepted steps */
    int64_t n_reject;    /* rejected step attempts */
    int64_t n_matvec;    /* generator applications */
    int64_t n_breakdown; /* happy breakdowns */
    double t_now;        /* time reached */
    double last_err;     /* last local error estimate */
} cufsp_expv_stats;

/* Generic matvec for the MVFun constructor form (src/KryExpvFSP.h:15): y += A x into a
 * zeroed y, device pointers, ordered on `stream`.  Return 0 on success. */
typedef int (*cufsp_matvec_fn)(const double *x, double *y, void *user, cufsp_stream_t stream);

/* n: vector length; m: Krylov dimension (1..60); tol; iop / q_iop: incomplete orthogonalisation
 * against the last q_iop vectors; anorm: the ||A|| estimate of the reference (default 1.0). */
cufsp_status cufsp_expv_create(int64_t n, int m, double tol, int iop, int q_iop, double anorm,
                               cufsp_expv **out);
cufsp_status cufsp_expv_destroy(cufsp_expv *E);
/* max_nstep (reference default 10000) and max_reject (reference default 1000), KryExpvFSP.h:68-69 */
cufsp_status cufsp_expv_set_limits(cufsp_expv *E, int64_t max_nstep, int64_t max_reject);
/* Bind the operator: a generator (evaluated at time t_mat with its tcoef) or a callback. */
cufsp_status cufsp_expv_bind_mat(cufsp_expv *E, cufsp_mat *A, double t_mat);
cufsp_status cufsp_expv_bind_matvec(cufsp_expv *E, cufsp_matvec_fn fn, void *user);
/* Bind the operator with explicit per-reaction coefficients (host, n_reactions doubles). */
cufsp_status cufsp_expv_bind_mat_coefs(cufsp_expv *E, cufsp_mat *A, const double *coefs);
/* KryExpvFSP::solve / step / reset_time / final_time_reached, KryExpvFSP.h:80-101.
 * v: device vector (in: start vector, out: exp(t_final A) v).  Synchronous per step. */
cufsp_status cufsp_expv_set_final_time(cufsp_expv *E, double t_final);
cufsp_status cufsp_expv_solve(cufsp_expv *E, double *v, cufsp_stream_t stream, cufsp_expv_stats *stats);
cufsp_status cufsp_expv_step(cufsp_expv *E, double *v, cufsp_stream_t stream);
cufsp_status cufsp_expv_reset_time(cufsp_expv *E);
cufsp_status cufsp_expv_final_time_reached(const cufsp_expv *E, int *reached);
cufsp_status cufsp_expv_get_stats(const cufsp_expv *E, cufsp_expv_stats *stats);

/* ---- BDF integrator for time-varying generators ------------------------------------------
 * Replaces the SUNDIALS CVODE path the reference drives through FSPMat::action: CVodeCreate(
 * CV_BDF, CV_NEWTON) with the matrix-free SPBCGS solver, RHS f(t,u) = A(t) u and J v = A(t) v
 * (tests/test_sundials.cu:67-91, 142-200; problems/hog1p_5species.cu:203-228, 287-336).
 * Variable order 1..5, quasi-constant step in backward-difference form, one GMRES solve of
 * (I - c A(t_new)) d = rhs per step (the CME is linear), error weights
 * 1 / (atol + rtol |p_i|) in the RMS norm (CVODE's), output times hit exactly (CVODE's tstop).
 * All vectors stay on the device; the step control runs on the host, synchronous per step.
 *
 *   create:  coefs (host, n_reactions doubles) freezes c_r; NULL evaluates A's tcoef(t) at
 *            every generator application (time-varying rates).  maxl: GMRES dimension, 1..60.
 *   init:    t0 and the initial distribution (copied; the caller keeps d_p0).
 *   advance: integrate to t_out and write p(t_out) to d_p.  one_step != 0 returns after one
 *            internal step toward t_out (CV_ONE_STEP) with the time reached in *t_reached.
 *   Errors: STEP_LIMIT when max_steps accepted steps do not reach t_out or the step size
 *   underflows; NONFINITE when the solution or a coefficient stops being finite. */
typedef struct cufsp_bdf_s cufsp_bdf;
typedef struct {
    double t;           /* time reached */
    double h;           /* next step size */
    double last_err;    /* weighted local error estimate of the last accepted step */
    int order;          /* current BDF order */
    int pad;
    int64_t n_steps;    /* accepted steps since init */
    int64_t n_reject;   /* steps rejected by the local error test */
    int64_t n_matvec;   /* generator applications */
    int64_t n_lin_iters;/* GMRES iterations */
    int64_t n_lin_fail; /* GMRES solves that did not converge (step halved) */
} cufsp_bdf_stats;
cufsp_status cufsp_bdf_create(cufsp_mat *A, const double *coefs, double rtol, double atol, int maxl,
                              cufsp_bdf **out);
cufsp_status cufsp_bdf_destroy(cufsp_bdf *B);
/* eps_lin: GMRES residual target in the weighted RMS norm (default 0.005); h_init <= 0: automatic
 * starting step; h_max <= 0: unbounded; max_steps: accepted steps per init (default 10^6). */
cufsp_status cufsp_bdf_set_options(cufsp_bdf *B, double eps_lin, double h_init, double h_max, int64_t max_steps);
/* Replace the frozen coefficients (NULL: use A's tcoef(t)); takes effect at the next init. */
cufsp_status cufsp_bdf_set_coefs(cufsp_bdf *B, const double *coefs);
cufsp_status cufsp_bdf_init(cufsp_bdf *B, double t0, const double *d_p0, cufsp_stream_t stream);
cufsp_status cufsp_bdf_advance(cufsp_bdf *B, double t_out, double *d_p, int one_step, cufsp_stream_t stream,
                               double *t_reached);
cufsp_status cufsp_bdf_get_stats(const cufsp_bdf *B, cufsp_bdf_stats *stats);

/* ---- FSP solver through output times ------------------------------------------------------
 * Replaces cme::FSPSolver (src/FSPSolver.h:16-111, src/FSPSolver.cpp:9-22; never compiled in the
 * reference, semantics defined here): next_time() advances the caller's device vector p from the
 * current time to the next output time with the Krylov exponential of the time-invariant
 * generator (coefs: host, n_reactions doubles, or NULL for tcoef(0)); solve() goes to the last
 * time; reset_time() returns to t = 0 keeping the vector.  After each advance the FSP truncation
 * error sum(p(0)) - sum(p(t)) is reported and compared with fsp_tol (stored, unused, in the
 * reference: FSPSolver.h:28).  Synchronous. */
typedef struct {
    int time_index;       /* index of the output time reached */
    double t;             /* time reached */
    double fsp_error;     /* probability that left the FSP box so far */
    int fsp_tol_exceeded; /* fsp_error > fsp_tol */
    int64_t krylov_steps; /* cumulative Krylov steps */
    int64_t matvecs;      /* cumulative generator applications */
} cufsp_solver_status;
typedef struct cufsp_solver_s cufsp_solver;
cufsp_status cufsp_solver_create(cufsp_mat *A, const double *times, int n_times, double fsp_tol,
                                 const double *coefs, double kry_tol, int m, int iop, int q_iop,
                                 cufsp_solver **out);
/* The same solver integrating with the BDF method (cufsp_bdf_*): coefs NULL follows A's tcoef(t)
 * (time-varying rates).  The caller's vector is read at the first advance after create,
 * reset_time or set_coefs (set_coefs(NULL) returns to tcoef(t)); krylov_steps then counts BDF steps. */
cufsp_status cufsp_solver_create_bdf(cufsp_mat *A, const double *times, int n_times, double fsp_tol,
                                     const double *coefs, double rtol, double atol, cufsp_solver **out);
cufsp_status cufsp_solver_destroy(cufsp_solver *S);
cufsp_status cufsp_solver_set_coefs(cufsp_solver *S, const double *coefs);
cufsp_status cufsp_solver_next_time(cufsp_solver *S, double *d_p, cufsp_stream_t stream, cufsp_solver_status *status);
cufsp_status cufsp_solver_solve(cufsp_solver *S, double *d_p, cufsp_stream_t stream, cufsp_solver_status *status);
cufsp_status cufsp_solver_reset_time(cufsp_solver *S);

/* ---- FSP with an adaptively grown box --------------------------------------------------------
 * No counterpart in the reference: cme::FSPSolver stores fsp_tol but never uses it
 * (src/FSPSolver.h:28).  The solver owns its distribution, since the box grows.  next_time() accepts
 * the interval ending at times[i] only if the FSP error sum p(0) - sum p(times[i]) is at most
 * fsp_tol * times[i] / times[last]; otherwise species whose upper face carries at least a tenth of
 * the largest face mass grow by the factor `grow` (up to max_bounds), the generator is rebuilt from
 * desc->prop_factor (required; evaluated on the host for every box), the distribution accepted at
 * the previous output time is embedded and the interval is solved again (Krylov: m, kry_tol).
 * When every species is at its maximum the solution is kept and fsp_tol_exceeded is set.
 * coefs: host, n_reactions time-invariant rates.  Synchronous. */
typedef struct {
    int time_index;        /* output time reached */
    double t;
    double fsp_error;      /* probability that left the box by t */
    int fsp_tol_exceeded;  /* the error is above its budget (box at its maximum) */
    int expansions;        /* box enlargements so far */
    int64_t n_states;      /* states of the current box */
    int bounds[16];        /* current box (first n_species entries) */
} cufsp_adaptive_status;
typedef struct cufsp_adaptive_s cufsp_adaptive;
cufsp_status cufsp_adaptive_create(const cufsp_model_desc *desc, const int *max_bounds, double grow, double fsp_tol,
                                   const double *coefs, const double *times, int n_times, double kry_tol, int m,
                                   cufsp_adaptive **out);
cufsp_status cufsp_adaptive_destroy(cufsp_adaptive *S);
/* d_p0: device, in the initial box (desc->fsp_bounds) */
cufsp_status cufsp_adaptive_set_initial(cufsp_adaptive *S, const double *d_p0, cufsp_stream_t stream);
cufsp_status cufsp_adaptive_next_time(cufsp_adaptive *S, cufsp_stream_t stream, cufsp_adaptive_status *status);
/* The current distribution (device, owned by the solver, valid until the next call), box and size. */
cufsp_status cufsp_adaptive_solution(const cufsp_adaptive *S, const double **d_p, int *bounds, int64_t *n_states);

/* ---- likelihood and data generation ----------------------------------------------------------
 * One time point of Likelihood::evaluate (src/Likelihood.cpp:14-21):
 *   *out = sum_k counts[k] * log(max(1e-44, q[k])),  q[k] = sum_{j<block} p[k*block + j],
 * i.e. p marginalised over the fastest-varying species whose index range has `block` states
 * (block = 1: no marginalisation).  d_p, d_counts: device, n and n/block doubles.  Synchronous. */
cufsp_status cufsp_loglik(int64_t n, const double *d_p, int64_t block, const double *d_counts, double *out,
                          cufsp_stream_t stream);
/* Likelihood::evaluate (src/Likelihood.cpp:8-33) in one call:
 *   *logL = sum_i sum_k counts_i[k] log max(1e-44, q_i[k]),  q_i = block sums of exp(times[i] A(c)) p0,
 * the Krylov solve (m, tol as cufsp_expv_create) carrying p through the data times on the device and
 * every time's term reduced there.  coefs: host, n_reactions (NULL: A's tcoef(0)); times: host,
 * non-decreasing; d_p0: device, n states (not modified); d_counts: device, n_times x n / block;
 * *fsp_error (nullable): sum p0 - sum p(times[last]), the FSP truncation error.  Synchronous. */
cufsp_status cufsp_likelihood_eval(cufsp_mat *A, const double *coefs, int n_times, const double *times,
                                   const double *d_p0, int64_t block, const double *d_counts, int m, double tol,
                                   double *logL, double *fsp_error, cufsp_stream_t stream);
/* Gradient of the log-likelihood above over several data times by the adjoint method (no counterpart
 * in the reference; its Likelihood has no gradient):
 *   log L(c) = sum_i sum_k counts_i[k] log max(1e-44, q_i[k]),  q_i = block sums of exp(times[i] A(c)) p0,
 *   grad[r] = d log L / d log c_r  (host, n_reactions),  *logL (host).
 * A: a KRONECKER generator (its transposed action is used); coefs (host, n_reactions) are the rates
 * c_r of the time-invariant A(c) = sum_r c_r A_r; times (host, n_times, non-decreasing, > 0);
 * d_p0 (device, n states); d_counts (device, n_times x n / block).  The forward Krylov solve (m, tol
 * as cufsp_expv_create) keeps p at every step boundary; the backward pass integrates the adjoint with
 * the transposed generator and accumulates int lambda^T A_r p ds exactly within the two Krylov
 * subspaces of every step.  Synchronous. */
cufsp_status cufsp_likelihood_grad(cufsp_mat *A, const double *coefs, int n_times, const double *times,
                                   const double *d_p0, int64_t block, const double *d_counts, int m, double tol,
                                   double *logL, double *grad, cufsp_stream_t stream);
/* The same gradient for n_sets parameter sets (coefs: host [n_sets][n_reactions]; logL: host [n_sets];
 * grad: host [n_sets][n_reactions]) sharing times, p0 and counts.  `workers` host threads, each with
 * its own KRONECKER generator built from desc, stream and workspaces, overlap their solves on the
 * GPU.  The workers' streams are non-blocking: the call first waits for the work queued on the
 * legacy default stream (the usual producer of d_p0 and d_counts); inputs written on other streams
 * must be complete before the call.  No counterpart in the reference.  Synchronous. */
cufsp_status cufsp_likelihood_grad_batched(const cufsp_model_desc *desc, int n_sets, const double *coefs,
                                           int n_times, const double *times, const double *d_p0, int64_t block,
                                           const double *d_counts, int m, double tol, int workers, double *logL,
                                           double *grad);
/* generate_data (src/Likelihood.cpp:35-84): Gillespie direct method from x0 (host, n_species
 * ints), an independent trajectory per (time, cell) as single-cell snapshots are, Philox streams
 * seeded by `seed`.  Propensities c_r * prod_s f_{r,s}(x_s) from the model's factor tables
 * (counts beyond the box use the table's edge value); coefs: host, or NULL for tcoef(0).
 * d_out: device int[n_times][n_cells][n_species].  CUFSP_ERR_STEP_LIMIT when a trajectory needs
 * more than max_events reactions.  Synchronous. */
cufsp_status cufsp_ssa(const cufsp_model_desc *desc, const double *coefs, const int *x0, const double *times,
                       int n_times, int n_cells, unsigned long long seed, int64_t max_events, int *d_out,
                       cufsp_stream_t stream);

/* ---- batched exp(tA)p over many instances, one persistent launch ---------------------------
 * No counterpart in the reference, which solves one instance per KryExpvFSP object; this is the
 * batched form of KryExpvFSP::solve (src/KryExpvFSP.cu:184-188) for parameter sweeps and
 * likelihood evaluations.  Instances share one reaction network (stoichiometry) but each has its
 * own box, factor tables and rate coefficients.  The whole adaptive Krylov solve -- Arnoldi, the
 * Pade exponential of the small Hessenberg matrix and the Expokit step control -- runs on the
 * device, one thread-block cluster per instance at a time, replayed as a CUDA graph.
 *   create:  fsp_bounds [n_instances][n_species]; factor_tables[i] -> n_reactions * sum_s (b_s + 1)
 *            doubles in the reference layout (as cufsp_model_desc); coefs [n_instances][n_reactions].
 *            m <= 32; iop / q_iop: incomplete orthogonalisation as in cufsp_expv_create.
 *   layout:  offsets (host, n_instances + 1): instance i's vector occupies
 *            [offsets[i], offsets[i] + n_i) of the packed device array; offsets[n] = total length.
 *   solve:   d_packed in: p(0) of every instance, out: exp(t_final A_i) p_i(0).  The first solve
 *            chooses the launch shape (autotuner, cached per device and network) unless
 *            cufsp_batch_set_shape fixed it.  Synchronous; stats (host, n_instances, or NULL).
 *            Returns STEP_LIMIT / NONFINITE if any instance failed (see its stat.status). */
typedef struct {
    int n_species;
    int n_reactions;
    const int *stoich_vals;
    const int *stoich_colidxs;
    const int *stoich_rowptrs;
    int n_instances;
    const int *fsp_bounds;
    const double *const *factor_tables;
    const double *coefs;
} cufsp_batch_desc;
typedef struct {
    double t;        /* time reached */
    double err;      /* last local error estimate */
    int steps;       /* accepted Krylov steps */
    int rejects;     /* rejected step sizes */
    int matvecs;     /* generator applications */
    int status;      /* 0 ok, 1 step limit, 2 NaN/Inf */
} cufsp_batch_stat;
typedef struct cufsp_batch_s cufsp_batch;
cufsp_status cufsp_batch_create(const cufsp_batch_desc *desc, int m, double tol, int iop, int q_iop, cufsp_batch **out);
cufsp_status cufsp_batch_destroy(cufsp_batch *B);
cufsp_status cufsp_batch_layout(const cufsp_batch *B, int64_t *offsets);
cufsp_status cufsp_batch_set_coefs(cufsp_batch *B, const double *coefs);
cufsp_status cufsp_batch_set_limits(cufsp_batch *B, int max_steps, int max_reject);
/* Fix the launch shape (CTAs per cluster 1..16, threads 128/256/512); (0, 0) re-enables the autotuner. */
cufsp_status cufsp_batch_set_shape(cufsp_batch *B, int cluster_ctas, int threads);
cufsp_status cufsp_batch_solve(cufsp_batch *B, double t_final, double *d_packed, cufsp_stream_t stream,
                               cufsp_batch_stat *stats);
cufsp_status cufsp_batch_describe(const cufsp_batch *B, char *buf, size_t len);

/* Dense exponential of a k x k column-major host matrix by scaling-and-squaring Pade(13,13)
 * (replaces arma::expmat at src/KryExpvFSP.cu:125). */
cufsp_status cufsp_expm_host(int k, const double *A, double *F);
/* The same for a block upper-triangular (k1 + k2) x (k1 + k2) matrix [[A11, A12], [0, A22]] (the
 * lower-left block of A is not read; F's is zero), three block products per matrix product instead
 * of eight.  The adjoint gradient's Van Loan exponentials have this form.  No counterpart in the
 * reference. */
cufsp_status cufsp_expm_blocktri_host(int k1, int k2, const double *A, double *F);

/* ---- vector helpers (device) ------------------------------------------------------------- */
/* sum of x (deterministic order); result written to host *out; synchronises `stream`. */
cufsp_status cufsp_vec_sum(int64_t n, const double *x, double *out, cufsp_stream_t stream);

/* Device buffers of released Krylov, adjoint and persistent-pass workspaces are kept in a per-process
 * cache for reuse (up to CUFSP_CACHE_MAX_MB megabytes, default 1024, read once from the environment);
 * an allocation of this library that runs out of memory returns that device's idle buffers and
 * retries.  This returns every idle buffer of every device to the driver now (e.g. before a caller's
 * own large allocation); *freed_bytes (nullable) receives the amount.  No counterpart in the reference. */
cufsp_status cufsp_cache_trim(size_t *freed_bytes);

/* d_dst[0..n) = d_src[0..n) (device to device), ordered on `stream`. */
cufsp_status cufsp_vec_copy(int64_t n, const double *d_src, double *d_dst, cufsp_stream_t stream);

/* Sum of the n doubles at x (device), written to the device double *d_out, with NO device memory
 * allocated: no counterpart in the reference.  It is meant for callers that cannot call cudaMalloc
 * themselves or let a library do it -- a framework or serving runtime that owns all device memory
 * through its own pool and accounts for every byte, or a code path that must not take the device
 * synchronisation that cudaMalloc/cudaFree can imply.
 * Limits and sharing: the scratch is a fixed 8 KB __device__ array in this library (one partial sum
 * per 4096-element block), held on every GPU that loads the library until the process exits, so
 * n <= CUFSP_NOALLOC_MAX_N; larger n returns CUFSP_ERR_INVALID_ARG.  The first call on a device looks
 * the array's address up (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  All calls share the array: calls that overlap on the GPU (other
 * streams, other host threads) race and must be serialised.  Asynchronous on `stream`; the
 * summation order is fixed, so the result is reproducible. */
#define CUFSP_NOALLOC_MAX_N 4194304
cufsp_status cufsp_vec_sum_noalloc(int64_t n, const double *x, double *d_out, cufsp_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* CUFSP_H */
