// cufsp_adaptive.cu -- FSP with an adaptively grown box (no counterpart in the reference: cme::FSPSolver
// stores fsp_tol but never uses it, src/FSPSolver.h:28).
//
// The FSP approximation loses exactly the probability that flows out of the box, so
// eps(t) = sum p(0) - sum p(t) bounds the error of the truncated solution in 1-norm.  The solver
// advances through output times t_1 < ... < t_K with the Krylov exponential and accepts the interval
// ending at t_i only if eps(t_i) <= fsp_tol * t_i / t_K (the budget grows with time, so the final error
// is at most fsp_tol).  Otherwise the box grows -- species whose upper face carries at least a tenth
// of the largest face mass, each by the factor `grow` up to its maximum -- the generator is rebuilt
// from the host factor function for the new box, the distribution accepted at t_{i-1} is embedded
// (same states, zeros elsewhere), and the interval is solved again.  The solver owns its vector,
// since the box size changes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "cufsp_internal.h"
#include "cufsp_reduce.cuh"

namespace cufsp {
namespace {

constexpr int kMaxS = CUFSP_MAX_SPECIES;

struct EmbedArgs {
    int ns;
    int64_t n_old;
    int dims_old[kMaxS];
    int64_t stride_new[kMaxS];
};

// p_new[idx_new(x)] = p_old[idx_old(x)] for every state x of the old box (p_new zeroed first).
__global__ void k_embed(const EmbedArgs a, const double *__restrict__ p_old, double *__restrict__ p_new) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n_old; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t rem = i, j = 0;
        for (int s = 0; s < a.ns; ++s) {
            const int64_t xs = rem % a.dims_old[s];
            rem /= a.dims_old[s];
            j += xs * a.stride_new[s];
        }
        p_new[j] = p_old[i];
    }
}

struct FaceArgs {
    int ns;
    int64_t n;
    int dims[kMaxS];
};

// mass on the upper face x_s = b_s of every species (ns outputs, deterministic reduction)
__global__ void __launch_bounds__(kRedThreads) k_face_mass(const FaceArgs a, const double *__restrict__ p,
                                                           double *__restrict__ out, double *__restrict__ partials,
                                                           unsigned int *__restrict__ counter) {
    __shared__ RedSmem<kMaxS> sm;
    double acc[kMaxS];
#pragma unroll
    for (int s = 0; s < kMaxS; ++s) acc[s] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t rem = i;
        const double v = p[i];
#pragma unroll
        for (int s = 0; s < kMaxS; ++s) {
            if (s < a.ns) {
                const int64_t xs = rem % a.dims[s];
                rem /= a.dims[s];
                if (xs == a.dims[s] - 1) acc[s] += fabs(v);
            }
        }
    }
    if (!grid_reduce<kMaxS>(acc, a.ns, partials, counter, sm)) return;
    for (int s = threadIdx.x; s < a.ns; s += blockDim.x) out[s] = sm.final_[s];
}

}  // namespace
}  // namespace cufsp

using namespace cufsp;

struct cufsp_adaptive_s {
    cufsp_model_desc desc;                 // copy (pointers into the vectors below)
    std::vector<int> sv, sc, sr, bounds, max_bounds;
    std::vector<double> coefs, times;
    double grow = 1.5, fsp_tol = 1e-6, kry_tol = 1e-8, mass0 = 1.0;
    int m = 30, index = 0, expansions = 0;
    double t_now = 0.0;
    cufsp_mat *A = nullptr;
    cufsp_expv *E = nullptr;
    double *p = nullptr, *p_prev = nullptr, *d_red = nullptr;
    int64_t n = 0;
    ReduceScratch rs;
    bool ready = false;
};

namespace {

void release_box(cufsp_adaptive *S) {
    if (S->E) cufsp_expv_destroy(S->E);
    if (S->A) cufsp_mat_destroy(S->A);
    if (S->p) cudaFree(S->p);
    if (S->p_prev) cudaFree(S->p_prev);
    S->E = nullptr;
    S->A = nullptr;
    S->p = S->p_prev = nullptr;
}

// Generator, Krylov driver and vectors for the current bounds.
cufsp_status build_box(cufsp_adaptive *S) {
    S->desc.fsp_bounds = S->bounds.data();
    cufsp_status s = cufsp_mat_create(&S->desc, CUFSP_FORMAT_KRONECKER, &S->A);
    if (s == CUFSP_SUCCESS) s = cufsp_mat_num_states(S->A, &S->n);
    if (s == CUFSP_SUCCESS) s = cufsp_expv_create(S->n, S->m, S->kry_tol, 0, 2, 1.0, &S->E);
    if (s == CUFSP_SUCCESS) s = cufsp_expv_bind_mat_coefs(S->E, S->A, S->coefs.data());
    if (s != CUFSP_SUCCESS) return s;
    if (dev_malloc(&S->p, sizeof(double) * S->n) != cudaSuccess ||
        dev_malloc(&S->p_prev, sizeof(double) * S->n) != cudaSuccess) {
        cudaGetLastError();
        return set_error(CUFSP_ERR_ALLOC, "adaptive FSP: vector allocation failed");
    }
    return CUFSP_SUCCESS;
}

cufsp_status sum_of(cufsp_adaptive *S, const double *v, cudaStream_t st, double *out) {
    cufsp_status s = launch_sum(S->n, v, S->d_red, S->rs, st);
    if (s != CUFSP_SUCCESS) return s;
    CUFSP_CUDA_TRY(cudaMemcpyAsync(out, S->d_red, sizeof(double), cudaMemcpyDeviceToHost, st));
    CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
    return CUFSP_SUCCESS;
}

// Grow the box in the directions that carry boundary mass of `v` (the rejected solution); embed the
// accepted distribution p_prev into the new box.  false when every species is at its maximum.
cufsp_status expand(cufsp_adaptive *S, const double *v, cudaStream_t st, bool *grown) {
    const int ns = S->desc.n_species;
    FaceArgs fa;
    std::memset(&fa, 0, sizeof(fa));
    fa.ns = ns;
    fa.n = S->n;
    for (int s = 0; s < ns; ++s) fa.dims[s] = S->bounds[s] + 1;
    const int grid = stream_grid(S->n, 4, std::min(device_info().sm_count * 4, S->rs.max_ctas));
    k_face_mass<<<grid, kRedThreads, 0, st>>>(fa, v, S->d_red, S->rs.partials, S->rs.counter);
    CUFSP_CUDA_TRY(cudaGetLastError());
    std::vector<double> face(ns);
    CUFSP_CUDA_TRY(cudaMemcpyAsync(face.data(), S->d_red, sizeof(double) * ns, cudaMemcpyDeviceToHost, st));
    CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
    double fmax = 0.0;
    for (int s = 0; s < ns; ++s)
        if (S->bounds[s] < S->max_bounds[s]) fmax = std::max(fmax, face[s]);
    std::vector<int> nb = S->bounds;
    bool any = false;
    for (int s = 0; s < ns; ++s) {
        if (S->bounds[s] >= S->max_bounds[s]) continue;
        if (fmax > 0.0 ? face[s] >= 0.1 * fmax : true) {
            nb[s] = std::min(S->max_bounds[s], std::max(S->bounds[s] + 1, (int)std::ceil((S->bounds[s] + 1) * S->grow) - 1));
            any = true;
        }
    }
    *grown = any;
    if (!any) return CUFSP_SUCCESS;
    // keep the accepted distribution, rebuild for the new box, embed
    double *old = nullptr;
    const int64_t n_old = S->n;
    std::vector<int> old_dims(ns);
    for (int s = 0; s < ns; ++s) old_dims[s] = S->bounds[s] + 1;
    CUFSP_CUDA_TRY(dev_malloc(&old, sizeof(double) * n_old));
    CUFSP_CUDA_TRY(cudaMemcpyAsync(old, S->p_prev, sizeof(double) * n_old, cudaMemcpyDeviceToDevice, st));
    CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
    release_box(S);
    S->bounds = nb;
    cufsp_status s = build_box(S);
    if (s == CUFSP_SUCCESS) {
        EmbedArgs ea;
        std::memset(&ea, 0, sizeof(ea));
        ea.ns = ns;
        ea.n_old = n_old;
        int64_t stv = 1;
        for (int k = 0; k < ns; ++k) {
            ea.dims_old[k] = old_dims[k];
            ea.stride_new[k] = stv;
            stv *= S->bounds[k] + 1;
        }
        cudaError_t e = cudaMemsetAsync(S->p_prev, 0, sizeof(double) * S->n, st);
        if (e == cudaSuccess) {
            k_embed<<<stream_grid(n_old, 4, device_info().sm_count * 8), 256, 0, st>>>(ea, old, S->p_prev);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) s = cuda_error(e, "adaptive FSP: embed");
    }
    cudaFree(old);
    ++S->expansions;
    return s;
}

}  // namespace

extern "C" cufsp_status cufsp_adaptive_create(const cufsp_model_desc *desc, const int *max_bounds, double grow,
                                              double fsp_tol, const double *coefs, const double *times, int n_times,
                                              double kry_tol, int m, cufsp_adaptive **out) {
    clear_error();
    if (!out || !desc || !max_bounds || !coefs || !times || n_times < 1 || !desc->prop_factor || !desc->fsp_bounds)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_adaptive_create: bad argument (prop_factor is required)");
    if (!(grow > 1.0) || !(fsp_tol > 0.0))
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_adaptive_create: grow must be > 1 and fsp_tol > 0");
    *out = nullptr;
    const int ns = desc->n_species, nr = desc->n_reactions;
    if (ns < 1 || ns > CUFSP_MAX_SPECIES || nr < 1 || nr > CUFSP_MAX_REACTIONS)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_adaptive_create: species or reaction count out of range");
    for (int i = 0; i < n_times; ++i)
        if (!std::isfinite(times[i]) || times[i] <= 0.0 || (i && !(times[i] > times[i - 1])))
            return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_adaptive_create: times must be finite, > 0, increasing");
    cufsp_adaptive *S = new cufsp_adaptive();
    S->desc = *desc;
    S->desc.factor_tables = nullptr;  // tables are re-evaluated from prop_factor for every box
    S->desc.prop_device = nullptr;
    S->sr.assign(desc->stoich_rowptrs, desc->stoich_rowptrs + nr + 1);
    const int nnz = S->sr[nr];
    S->sv.assign(desc->stoich_vals, desc->stoich_vals + nnz);
    S->sc.assign(desc->stoich_colidxs, desc->stoich_colidxs + nnz);
    S->desc.stoich_vals = S->sv.data();
    S->desc.stoich_colidxs = S->sc.data();
    S->desc.stoich_rowptrs = S->sr.data();
    S->bounds.assign(desc->fsp_bounds, desc->fsp_bounds + ns);
    S->max_bounds.assign(max_bounds, max_bounds + ns);
    for (int s = 0; s < ns; ++s)
        if (S->max_bounds[s] < S->bounds[s]) S->max_bounds[s] = S->bounds[s];
    S->coefs.assign(coefs, coefs + nr);
    S->times.assign(times, times + n_times);
    S->grow = grow;
    S->fsp_tol = fsp_tol;
    S->kry_tol = kry_tol;
    S->m = m;
    cufsp_status s = build_box(S);
    if (s == CUFSP_SUCCESS) s = S->rs.init(device_info().sm_count * 4, CUFSP_MAX_SPECIES);
    if (s == CUFSP_SUCCESS && dev_malloc(&S->d_red, sizeof(double) * CUFSP_MAX_SPECIES) != cudaSuccess)
        s = set_error(CUFSP_ERR_ALLOC, "cufsp_adaptive_create: cudaMalloc");
    if (s != CUFSP_SUCCESS) {
        cufsp_adaptive_destroy(S);
        return s;
    }
    *out = S;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_adaptive_destroy(cufsp_adaptive *S) {
    if (!S) return CUFSP_SUCCESS;
    release_box(S);
    if (S->d_red) cudaFree(S->d_red);
    S->rs.release();
    delete S;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_adaptive_set_initial(cufsp_adaptive *S, const double *d_p0, cufsp_stream_t stream) {
    if (!S || !d_p0) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_adaptive_set_initial: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    CUFSP_CUDA_TRY(cudaMemcpyAsync(S->p, d_p0, sizeof(double) * S->n, cudaMemcpyDeviceToDevice, st));
    cufsp_status s = sum_of(S, S->p, st, &S->mass0);
    if (s != CUFSP_SUCCESS) return s;
    S->t_now = 0.0;
    S->index = 0;
    S->ready = true;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_adaptive_next_time(cufsp_adaptive *S, cufsp_stream_t stream, cufsp_adaptive_status *status) {
    if (!S) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_adaptive_next_time: NULL argument");
    if (!S->ready) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_adaptive_next_time: set the initial distribution first");
    if (S->index >= (int)S->times.size())
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_adaptive_next_time: all output times already reached");
    cudaStream_t st = (cudaStream_t)stream;
    const double t_end = S->times.back();
    const double target = S->times[S->index];
    const double budget = S->fsp_tol * target / t_end;
    CUFSP_CUDA_TRY(cudaMemcpyAsync(S->p_prev, S->p, sizeof(double) * S->n, cudaMemcpyDeviceToDevice, st));
    double err = 0.0;
    bool exceeded = false;
    for (int attempt = 0; attempt < 64; ++attempt) {
        cufsp_status s = cufsp_expv_set_final_time(S->E, target - S->t_now);
        if (s == CUFSP_SUCCESS) s = cufsp_expv_reset_time(S->E);
        if (s == CUFSP_SUCCESS) s = cufsp_expv_solve(S->E, S->p, stream, nullptr);
        double mass = 0.0;
        if (s == CUFSP_SUCCESS) s = sum_of(S, S->p, st, &mass);
        if (s != CUFSP_SUCCESS) return s;
        err = S->mass0 - mass;
        if (err <= budget) break;
        bool grown = false;
        s = expand(S, S->p, st, &grown);
        if (s != CUFSP_SUCCESS) return s;
        if (!grown) {  // every species is at its maximum: keep the solution, report the excess
            exceeded = true;
            break;
        }
        CUFSP_CUDA_TRY(cudaMemcpyAsync(S->p, S->p_prev, sizeof(double) * S->n, cudaMemcpyDeviceToDevice, st));
    }
    S->t_now = target;
    if (status) {
        status->time_index = S->index;
        status->t = target;
        status->fsp_error = err;
        status->fsp_tol_exceeded = exceeded || err > budget;
        status->expansions = S->expansions;
        status->n_states = S->n;
        for (int s = 0; s < S->desc.n_species && s < CUFSP_MAX_SPECIES; ++s) status->bounds[s] = S->bounds[s];
    }
    ++S->index;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_adaptive_solution(const cufsp_adaptive *S, const double **d_p, int *bounds, int64_t *n) {
    if (!S) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_adaptive_solution: NULL argument");
    if (d_p) *d_p = S->p;
    if (bounds) std::copy(S->bounds.begin(), S->bounds.end(), bounds);
    if (n) *n = S->n;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_vec_copy(int64_t n, const double *d_src, double *d_dst, cufsp_stream_t stream) {
    if (n < 0 || (n > 0 && (!d_src || !d_dst))) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_vec_copy: bad argument");
    if (n == 0) return CUFSP_SUCCESS;
    CUFSP_CUDA_TRY(cudaMemcpyAsync(d_dst, d_src, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice,
                                   (cudaStream_t)stream));
    return CUFSP_SUCCESS;
}
