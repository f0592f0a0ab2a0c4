// cufsp_stats.cu -- likelihood reduction and the stochastic simulation (SSA) data generator.
//
//  * cufsp_loglik: log L = sum_k counts[k] * log(max(1e-44, q[k])), q[k] = sum_{j<block} p[k*block+j]
//    -- the per-time term of Likelihood::evaluate (src/Likelihood.cpp:14-21: log(max(1e-44, p)))
//    with the marginalisation over the fastest-varying species (a contiguous block of the state
//    index) that single-cell data binned over a subset of species needs.  Deterministic order.
//  * cufsp_ssa: Gillespie's direct method, one thread per cell, counter-based Philox streams keyed
//    by (seed, cell) -- generate_data (src/Likelihood.cpp:35-84) with a reproducible seed.
#include <curand_kernel.h>

#include <cmath>
#include <vector>

#include "cufsp_internal.h"
#include "cufsp_reduce.cuh"

namespace cufsp {

__global__ void __launch_bounds__(kRedThreads) k_loglik(int64_t nk, int block, const double *__restrict__ p,
                                                       const double *__restrict__ counts, double *__restrict__ partials,
                                                       unsigned int *__restrict__ counter, double *__restrict__ out) {
    __shared__ RedSmem<1> sm;
    double acc[1] = {0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += stride) {
        const double c = counts[k];
        if (c != 0.0) {
            double q = 0.0;
            const double *pk = p + k * block;
            for (int j = 0; j < block; ++j) q += pk[j];
            acc[0] = fma(c, log(fmax(1e-44, q)), acc[0]);
        }
    }
    if (grid_reduce<1>(acc, 1, partials, counter, sm) && threadIdx.x == 0) out[0] = sm.final_[0];
}

struct SsaArgs {
    const double *__restrict__ tables;  // [nr][tab_stride] factor tables
    const int *__restrict__ nu;         // [nr][ns]
    const int *__restrict__ x0;         // [ns] initial state
    const double *__restrict__ times;   // [n_times] increasing output times
    int *__restrict__ out;              // [n_times][n_cells][ns]
    int *__restrict__ err;              // set when a cell exceeds max_events
    double coef[CUFSP_MAX_REACTIONS];
    int bounds_tab[CUFSP_MAX_SPECIES];  // table extents b_s (states beyond use the edge value)
    int tab_off[CUFSP_MAX_SPECIES];
    int ns, nr, tab_stride, n_cells, n_times;
    int64_t max_events;
    unsigned long long seed;
};

// Propensity from the factor tables; a species count beyond the tabulated box uses the last
// tabulated value (the tables are only known on the box).
__device__ __forceinline__ double ssa_prop(const SsaArgs &a, const int *x, int r) {
    double v = a.coef[r];
    const double *t = a.tables + (size_t)r * a.tab_stride;
    for (int s = 0; s < a.ns; ++s) {
        int xs = x[s];
        xs = xs < 0 ? 0 : (xs > a.bounds_tab[s] ? a.bounds_tab[s] : xs);
        v *= __ldg(t + a.tab_off[s] + xs);
    }
    return v;
}

// One independent trajectory per (output time, cell), as generate_data draws a fresh sample from
// x0 for every time point (src/Likelihood.cpp:43-73): single-cell snapshots are destructive.
__global__ void k_ssa(const SsaArgs a) {
    const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (int64_t)a.n_cells * a.n_times) return;
    const int it = (int)(gid / a.n_cells);
    const double t_end = a.times[it];
    curandStatePhilox4_32_10_t rng;
    curand_init(a.seed, (unsigned long long)gid, 0ull, &rng);
    int x[CUFSP_MAX_SPECIES];
    for (int s = 0; s < a.ns; ++s) x[s] = a.x0[s];
    double prop[CUFSP_MAX_REACTIONS];
    double t = 0.0;
    for (int64_t events = 0;; ++events) {
        double a0 = 0.0;
        for (int r = 0; r < a.nr; ++r) {
            prop[r] = ssa_prop(a, x, r);
            a0 += prop[r];
        }
        if (!(a0 > 0.0)) break;                         // absorbing state
        const double tau = -log(curand_uniform_double(&rng)) / a0;  // uniform on (0, 1]
        if (t + tau > t_end) break;                     // next event after the snapshot time
        if (events >= a.max_events) {
            atomicExch(a.err, 1);
            break;
        }
        const double u2 = curand_uniform_double(&rng) * a0;
        int r = 0;
        double acc = prop[0];
        while (acc < u2 && r < a.nr - 1) acc += prop[++r];
        for (int s = 0; s < a.ns; ++s) x[s] += a.nu[r * a.ns + s];
        t += tau;
    }
    int *o = a.out + (size_t)gid * a.ns;  // layout [n_times][n_cells][ns]
    for (int s = 0; s < a.ns; ++s) o[s] = x[s];
}

}  // namespace cufsp

using namespace cufsp;

extern "C" cufsp_status cufsp_loglik(int64_t n, const double *d_p, int64_t block, const double *d_counts,
                                     double *out, cufsp_stream_t stream) {
    if (!d_p || !d_counts || !out || n < 1 || block < 1 || n % block != 0 || block > 2147483647LL)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_loglik: bad argument");
    // scratch in order on the caller's stream: no device-wide synchronisation, so concurrent callers
    // on other streams (the batched gradient's workers) keep running
    cudaStream_t st = (cudaStream_t)stream;
    ReduceScratch rs;
    const int ctas = device_info().sm_count * 4;
    cufsp_status s = rs.init(ctas, 1, st);
    double *d_out = nullptr;
    if (s == CUFSP_SUCCESS && cache_alloc((void **)&d_out, sizeof(double)) != cudaSuccess)
        s = set_error(CUFSP_ERR_ALLOC, "cufsp_loglik: device allocation failed");
    if (s == CUFSP_SUCCESS) {
        const int64_t nk = n / block;
        const int g = stream_grid(nk, 1, ctas);
        k_loglik<<<g, kRedThreads, 0, (cudaStream_t)stream>>>(nk, (int)block, d_p, d_counts, rs.partials, rs.counter,
                                                             d_out);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, sizeof(double), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
        if (e != cudaSuccess) s = cuda_error(e, "cufsp_loglik");
    }
    if (d_out) cache_free(d_out, st);
    rs.release(st);
    return s;
}

// Likelihood::evaluate (src/Likelihood.cpp:8-33) as one call: the Krylov solve carries p(0) through
// the data times and every time's term is reduced on the device into its own slot; one device->host
// read at the end.  The solve is KryExpvFSP::solve between consecutive times (t_now carries over).
extern "C" cufsp_status cufsp_likelihood_eval(cufsp_mat *A, const double *coefs, int n_times, const double *times,
                                              const double *d_p0, int64_t block, const double *d_counts, int m,
                                              double tol, double *logL, double *fsp_error, cufsp_stream_t stream) {
    clear_error();
    if (!A || !times || !d_p0 || !d_counts || !logL || n_times < 1)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_likelihood_eval: NULL argument");
    int64_t n = 0;
    cufsp_mat_num_states(A, &n);
    if (block < 1 || n % block != 0 || block > 2147483647LL)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_likelihood_eval: bad block");
    for (int i = 0; i < n_times; ++i)
        if (!(times[i] >= (i ? times[i - 1] : 0.0)) || !std::isfinite(times[i]))
            return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_likelihood_eval: times must be finite and non-decreasing");
    cudaStream_t st = (cudaStream_t)stream;
    cufsp_expv *E = nullptr;
    cufsp_status s = cufsp_expv_create(n, m, tol, 0, 2, 1.0, &E);
    if (s == CUFSP_SUCCESS) {
        if (coefs) s = cufsp_expv_bind_mat_coefs(E, A, coefs);
        else s = cufsp_expv_bind_mat(E, A, 0.0);
    }
    double *p = nullptr, *d_ll = nullptr;
    ReduceScratch rs;
    const int ctas = device_info().sm_count * 4;
    if (s == CUFSP_SUCCESS && cache_alloc((void **)&p, sizeof(double) * (size_t)n) != cudaSuccess)
        s = set_error(CUFSP_ERR_ALLOC, "cufsp_likelihood_eval: device allocation failed");
    if (s == CUFSP_SUCCESS && cache_alloc((void **)&d_ll, sizeof(double) * (size_t)(n_times + 2)) != cudaSuccess)
        s = set_error(CUFSP_ERR_ALLOC, "cufsp_likelihood_eval: device allocation failed");
    if (s == CUFSP_SUCCESS) s = rs.init(ctas, 1);
    if (s == CUFSP_SUCCESS) {
        const cudaError_t e = cudaMemcpyAsync(p, d_p0, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) s = cuda_error(e, "cufsp_likelihood_eval");
    }
    // mass at t = 0 (for the FSP error)
    if (s == CUFSP_SUCCESS) s = launch_sum(n, p, d_ll + n_times, rs, st);
    const int64_t nk = n / block;
    for (int i = 0; i < n_times && s == CUFSP_SUCCESS; ++i) {
        s = cufsp_expv_set_final_time(E, times[i]);
        if (s == CUFSP_SUCCESS) s = cufsp_expv_solve(E, p, stream, nullptr);
        if (s != CUFSP_SUCCESS) break;
        const int g = stream_grid(nk, 1, ctas);
        k_loglik<<<g, kRedThreads, 0, st>>>(nk, (int)block, p, d_counts + (size_t)i * nk, rs.partials, rs.counter,
                                            d_ll + i);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) s = cuda_error(e, "cufsp_likelihood_eval");
    }
    if (s == CUFSP_SUCCESS) s = launch_sum(n, p, d_ll + n_times + 1, rs, st);
    std::vector<double> h(n_times + 2, 0.0);
    if (s == CUFSP_SUCCESS) {
        cudaError_t e = cudaMemcpyAsync(h.data(), d_ll, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) s = cuda_error(e, "cufsp_likelihood_eval");
    }
    if (s == CUFSP_SUCCESS) {
        double ll = 0.0;
        for (int i = 0; i < n_times; ++i) ll += h[i];  // time order, as the reference's loop
        *logL = ll;
        if (fsp_error) *fsp_error = h[n_times] - h[n_times + 1];
    }
    cudaStreamSynchronize(st);
    cufsp_expv_destroy(E);
    cache_free(p, st);
    cache_free(d_ll, st);
    rs.release(st);
    return s;
}

extern "C" cufsp_status cufsp_ssa(const cufsp_model_desc *desc, const double *coefs, const int *x0, const double *times,
                                  int n_times, int n_cells, unsigned long long seed, int64_t max_events, int *d_out,
                                  cufsp_stream_t stream) {
    ModelHost m;
    cufsp_status s = model_from_desc(desc, true, m);
    if (s != CUFSP_SUCCESS) return s;
    if (!x0 || !times || n_times < 1 || n_cells < 1 || !d_out || max_events < 1 || m.nr > CUFSP_MAX_REACTIONS)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_ssa: bad argument");
    for (int i = 1; i < n_times; ++i)
        if (!(times[i] > times[i - 1])) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_ssa: times must increase");
    std::vector<double> c(m.nr, 1.0);
    if (coefs) c.assign(coefs, coefs + m.nr);
    else if (m.tcoef) m.tcoef(0.0, c.data(), m.tcoef_user);  // generate_data uses t_fun(0, params)
    for (double v : c)
        if (!std::isfinite(v) || v < 0.0) return set_error(CUFSP_ERR_NONFINITE, "cufsp_ssa: rates must be finite and >= 0");
    SsaArgs a;
    a.ns = m.ns;
    a.nr = m.nr;
    a.tab_stride = m.tab_stride;
    a.n_cells = n_cells;
    a.n_times = n_times;
    a.max_events = max_events;
    a.seed = seed;
    for (int r = 0; r < CUFSP_MAX_REACTIONS; ++r) a.coef[r] = r < m.nr ? c[r] : 0.0;
    for (int sp = 0; sp < CUFSP_MAX_SPECIES; ++sp) {
        a.bounds_tab[sp] = sp < m.ns ? m.bounds[sp] : 0;
        a.tab_off[sp] = sp < m.ns ? m.tab_off[sp] : 0;
    }
    double *d_tab = nullptr, *d_times = nullptr;
    int *d_nu = nullptr, *d_x0 = nullptr, *d_err = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = dev_malloc(&d_tab, sizeof(double) * m.tables.size());
    if (e == cudaSuccess) e = dev_malloc(&d_nu, sizeof(int) * m.nu.size());
    if (e == cudaSuccess) e = dev_malloc(&d_x0, sizeof(int) * m.ns);
    if (e == cudaSuccess) e = dev_malloc(&d_times, sizeof(double) * n_times);
    if (e == cudaSuccess) e = dev_malloc(&d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(d_tab, m.tables.data(), sizeof(double) * m.tables.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_nu, m.nu.data(), sizeof(int) * m.nu.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_x0, x0, sizeof(int) * m.ns, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_times, times, sizeof(double) * n_times, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_err, 0, sizeof(int));
    if (e == cudaSuccess) e = upload_fence();
    int herr = 0;
    if (e == cudaSuccess) {
        a.tables = d_tab;
        a.nu = d_nu;
        a.x0 = d_x0;
        a.times = d_times;
        a.out = d_out;
        a.err = d_err;
        const int64_t total = (int64_t)n_cells * n_times;
        k_ssa<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(a);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    cudaFree(d_tab);
    cudaFree(d_nu);
    cudaFree(d_x0);
    cudaFree(d_times);
    cudaFree(d_err);
    if (e != cudaSuccess) return cuda_error(e, "cufsp_ssa");
    if (herr) return set_error(CUFSP_ERR_STEP_LIMIT, "cufsp_ssa: a cell exceeded max_events");
    return CUFSP_SUCCESS;
}
