// cufsp_solver.cu -- FSP time stepping through output times (replaces cme::FSPSolver,
// src/FSPSolver.h:16-111, src/FSPSolver.cpp:9-22, which never compiled in the reference).
//
// Semantics defined here (the reference only fixes the API): next_time() advances the caller's
// probability vector from the current time to the next output time, solve() to the last one,
// reset_time() returns to t = 0 (the vector is kept, as in the reference).  After every advance
// the FSP truncation error 1 - sum(p) -- the probability that left the box through the generator's
// boundary outflow -- is computed on the device and compared with fsp_tol (stored but unused by
// the reference, FSPSolver.h:28).  Time-invariant generators use the Krylov exponential (the
// coefficients c_r are taken at t = 0 or given explicitly); solvers made by
// cufsp_solver_create_bdf integrate with the BDF method instead, which also handles c_r(t), and
// read the caller's vector only at the first advance after create / reset_time / set_coefs.
#include <cmath>
#include <cstring>
#include <vector>

#include "cufsp_internal.h"

using namespace cufsp;

struct cufsp_solver_s {
    cufsp_mat *A = nullptr;
    cufsp_expv *E = nullptr;
    cufsp_bdf *B = nullptr;  // BDF path (time-varying rates); E is then unused
    bool bdf_ready = false;
    std::vector<double> times;
    double fsp_tol = 0.0;
    double t_now = 0.0;
    int index = 0;
    double mass0 = 1.0;  // sum(p) when the solver started from t = 0
    bool have_mass0 = false;
    double *d_sum = nullptr;
    ReduceScratch rs;
    cufsp_solver_status last;
};

namespace {

cufsp_status mass(cufsp_solver *S, const double *d_p, cudaStream_t st, double *out) {
    int64_t n = 0;
    cufsp_mat_num_states(S->A, &n);
    cufsp_status s = launch_sum(n, d_p, S->d_sum, S->rs, st);
    if (s != CUFSP_SUCCESS) return s;
    CUFSP_CUDA_TRY(cudaMemcpyAsync(out, S->d_sum, sizeof(double), cudaMemcpyDeviceToHost, st));
    CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
    return CUFSP_SUCCESS;
}

cufsp_status advance_to(cufsp_solver *S, double t_target, double *d_p, cudaStream_t st) {
    if (!S->have_mass0) {
        cufsp_status s = mass(S, d_p, st, &S->mass0);
        if (s != CUFSP_SUCCESS) return s;
        S->have_mass0 = true;
    }
    const double dt = t_target - S->t_now;
    if (S->B) {
        if (!S->bdf_ready) {
            cufsp_status s = cufsp_bdf_init(S->B, S->t_now, d_p, (cufsp_stream_t)st);
            if (s != CUFSP_SUCCESS) return s;
            S->bdf_ready = true;
        }
        cufsp_status s = cufsp_bdf_advance(S->B, t_target, d_p, 0, (cufsp_stream_t)st, nullptr);
        if (s != CUFSP_SUCCESS) {
            S->bdf_ready = false;
            return s;
        }
    } else if (dt > 0.0) {
        cufsp_status s = cufsp_expv_set_final_time(S->E, dt);
        if (s == CUFSP_SUCCESS) s = cufsp_expv_reset_time(S->E);
        if (s == CUFSP_SUCCESS) s = cufsp_expv_solve(S->E, d_p, (cufsp_stream_t)st, nullptr);
        if (s != CUFSP_SUCCESS) return s;
    }
    S->t_now = t_target;
    double m = 0.0;
    cufsp_status s = mass(S, d_p, st, &m);
    if (s != CUFSP_SUCCESS) return s;
    S->last.t = S->t_now;
    S->last.time_index = S->index;
    S->last.fsp_error = S->mass0 - m;
    S->last.fsp_tol_exceeded = S->last.fsp_error > S->fsp_tol;
    if (S->B) {
        cufsp_bdf_stats bs;
        cufsp_bdf_get_stats(S->B, &bs);
        S->last.krylov_steps = bs.n_steps;
        S->last.matvecs = bs.n_matvec;
    } else {
        cufsp_expv_stats es;
        cufsp_expv_get_stats(S->E, &es);
        S->last.krylov_steps = es.n_steps;
        S->last.matvecs = es.n_matvec;
    }
    return CUFSP_SUCCESS;
}

}  // namespace

namespace {

cufsp_status solver_new(cufsp_mat *A, const double *times, int n_times, double fsp_tol, cufsp_solver **out) {
    clear_error();
    if (!out || !A || !times || n_times < 1 || !(fsp_tol >= 0.0))
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_solver_create: bad argument");
    *out = nullptr;
    for (int i = 0; i < n_times; ++i) {
        if (!std::isfinite(times[i]) || times[i] < 0.0 || (i && !(times[i] > times[i - 1])))
            return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_solver_create: times must be finite, >= 0, increasing");
    }
    cufsp_solver *S = new cufsp_solver();
    S->A = A;
    S->times.assign(times, times + n_times);
    S->fsp_tol = fsp_tol;
    std::memset(&S->last, 0, sizeof(S->last));
    *out = S;
    return CUFSP_SUCCESS;
}

cufsp_status solver_finish(cufsp_solver *S, cufsp_status s, cufsp_solver **out) {
    if (s == CUFSP_SUCCESS) s = S->rs.init(device_info().sm_count * 4, 1);
    if (s == CUFSP_SUCCESS && dev_malloc(&S->d_sum, sizeof(double)) != cudaSuccess)
        s = set_error(CUFSP_ERR_ALLOC, "cufsp_solver_create: cudaMalloc");
    if (s != CUFSP_SUCCESS) {
        cufsp_solver_destroy(S);
        *out = nullptr;
        return s;
    }
    *out = S;
    return CUFSP_SUCCESS;
}

}  // namespace

extern "C" cufsp_status cufsp_solver_create_bdf(cufsp_mat *A, const double *times, int n_times, double fsp_tol,
                                                const double *coefs, double rtol, double atol, cufsp_solver **out) {
    cufsp_solver *S = nullptr;
    cufsp_status s = solver_new(A, times, n_times, fsp_tol, &S);
    if (s != CUFSP_SUCCESS) return s;
    s = cufsp_bdf_create(A, coefs, rtol, atol, 30, &S->B);
    return solver_finish(S, s, out);
}

extern "C" cufsp_status cufsp_solver_create(cufsp_mat *A, const double *times, int n_times, double fsp_tol,
                                            const double *coefs, double kry_tol, int m, int iop, int q_iop,
                                            cufsp_solver **out) {
    cufsp_solver *S = nullptr;
    cufsp_status s = solver_new(A, times, n_times, fsp_tol, &S);
    if (s != CUFSP_SUCCESS) return s;
    int64_t n = 0;
    cufsp_mat_num_states(A, &n);
    s = cufsp_expv_create(n, m, kry_tol, iop, q_iop, 1.0, &S->E);
    if (s == CUFSP_SUCCESS) s = coefs ? cufsp_expv_bind_mat_coefs(S->E, A, coefs) : cufsp_expv_bind_mat(S->E, A, 0.0);
    return solver_finish(S, s, out);
}

extern "C" cufsp_status cufsp_solver_destroy(cufsp_solver *S) {
    if (!S) return CUFSP_SUCCESS;
    cufsp_expv_destroy(S->E);
    cufsp_bdf_destroy(S->B);
    if (S->d_sum) cudaFree(S->d_sum);
    S->rs.release();
    delete S;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_solver_set_coefs(cufsp_solver *S, const double *coefs) {
    if (!S) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_solver_set_coefs: NULL argument");
    if (S->B) {
        S->bdf_ready = false;
        return cufsp_bdf_set_coefs(S->B, coefs);
    }
    if (!coefs) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_solver_set_coefs: NULL argument");
    return cufsp_expv_bind_mat_coefs(S->E, S->A, coefs);
}

// FSPSolver::next_time (src/FSPSolver.cpp:9-15)
extern "C" cufsp_status cufsp_solver_next_time(cufsp_solver *S, double *d_p, cufsp_stream_t stream,
                                               cufsp_solver_status *status) {
    if (!S || !d_p) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_solver_next_time: NULL argument");
    if (S->index >= (int)S->times.size())
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_solver_next_time: all output times already reached");
    cufsp_status s = advance_to(S, S->times[S->index], d_p, (cudaStream_t)stream);
    if (s != CUFSP_SUCCESS) return s;
    ++S->index;
    if (status) *status = S->last;
    return CUFSP_SUCCESS;
}

// FSPSolver::solve (src/FSPSolver.cpp:17-22): to the last output time
extern "C" cufsp_status cufsp_solver_solve(cufsp_solver *S, double *d_p, cufsp_stream_t stream,
                                           cufsp_solver_status *status) {
    if (!S || !d_p) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_solver_solve: NULL argument");
    S->index = (int)S->times.size() - 1;
    cufsp_status s = advance_to(S, S->times.back(), d_p, (cudaStream_t)stream);
    if (s != CUFSP_SUCCESS) return s;
    S->index = (int)S->times.size();
    if (status) *status = S->last;
    return CUFSP_SUCCESS;
}

// FSPSolver::reset_time (src/FSPSolver.h:103-109): back to t = 0, the vector is the caller's
extern "C" cufsp_status cufsp_solver_reset_time(cufsp_solver *S) {
    if (!S) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_solver_reset_time: NULL argument");
    S->index = 0;
    S->t_now = 0.0;
    S->have_mass0 = false;
    S->bdf_ready = false;
    return CUFSP_SUCCESS;
}
