// cufsp_vec.cu -- multi-vector streaming primitives with deterministic reductions, shared by the
// BDF integrator and its GMRES linear solver.  Each kernel streams its vectors once; reductions
// finish in the last CTA (grid_reduce), so results do not depend on CTA scheduling.
#include <algorithm>
#include <cmath>

#include "cufsp_internal.h"
#include "cufsp_reduce.cuh"
#include "cufsp_vec.h"

namespace cufsp {

namespace {

struct VecArgs {
    const double *vec[kVecMaxK];
    double c[kVecMaxK];  // host coefficients (lincomb)
    const double *dc;    // device coefficients (maxpy)
    double *q;           // in/out vector
    const double *w;     // weights, nullable
    int64_t n;
    int K;
    bool accumulate;
    double *d_out;
    double *partials;
    unsigned int *counter;
};

__device__ __forceinline__ double wsq(const double *w, int64_t i) {
    if (!w) return 1.0;
    const double x = __ldg(w + i);
    return x * x;
}

// d_out[k] = sum_i vec[k][i] q[i] w[i]^2
template <int KP>
__global__ void __launch_bounds__(kRedThreads) k_wdot(const VecArgs a) {
    __shared__ RedSmem<KP> sm;
    double acc[KP];
#pragma unroll
    for (int k = 0; k < KP; ++k) acc[k] = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const double qi = a.q[i] * wsq(a.w, i);
#pragma unroll
        for (int k = 0; k < KP; ++k)
            if (k < a.K) acc[k] = fma(__ldg(a.vec[k] + i), qi, acc[k]);
    }
    if (!grid_reduce<KP>(acc, a.K, a.partials, a.counter, sm)) return;
    for (int k = threadIdx.x; k < a.K; k += blockDim.x) a.d_out[k] = sm.final_[k];
}

// q -= sum_k dc[k] vec[k];  d_out[0] = ||q||_w
template <int KP>
__global__ void __launch_bounds__(kRedThreads) k_maxpy_wnorm(const VecArgs a) {
    __shared__ RedSmem<1> sm;
    __shared__ double cs[KP];
    for (int k = threadIdx.x; k < KP; k += blockDim.x) cs[k] = k < a.K ? a.dc[k] : 0.0;
    __syncthreads();
    double acc[1] = {0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        double qi = a.q[i];
#pragma unroll
        for (int k = 0; k < KP; ++k)
            if (k < a.K) qi = fma(-cs[k], __ldg(a.vec[k] + i), qi);
        a.q[i] = qi;
        acc[0] = fma(qi * qi, wsq(a.w, i), acc[0]);
    }
    if (grid_reduce<1>(acc, 1, a.partials, a.counter, sm) && threadIdx.x == 0) a.d_out[0] = sqrt(sm.final_[0]);
}

// q = (accumulate ? q : 0) + sum_k c[k] vec[k];  d_out[0] = ||q||_w when d_out
template <int KP>
__global__ void __launch_bounds__(kRedThreads) k_lincomb(const VecArgs a) {
    __shared__ RedSmem<1> sm;
    double acc[1] = {0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        double s = a.accumulate ? a.q[i] : 0.0;
#pragma unroll
        for (int k = 0; k < KP; ++k)
            if (k < a.K) s = fma(a.c[k], a.vec[k][i], s);
        a.q[i] = s;
        acc[0] = fma(s * s, wsq(a.w, i), acc[0]);
    }
    if (!a.d_out) return;
    if (grid_reduce<1>(acc, 1, a.partials, a.counter, sm) && threadIdx.x == 0) a.d_out[0] = sqrt(sm.final_[0]);
}

// d_out[0] = ||q||_w
__global__ void __launch_bounds__(kRedThreads) k_wnorm(const VecArgs a) {
    __shared__ RedSmem<1> sm;
    double acc[1] = {0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const double x = a.q[i];
        acc[0] = fma(x * x, wsq(a.w, i), acc[0]);
    }
    if (grid_reduce<1>(acc, 1, a.partials, a.counter, sm) && threadIdx.x == 0) a.d_out[0] = sqrt(sm.final_[0]);
}

__global__ void __launch_bounds__(256) k_normalize(int64_t n, double *v, const double *d_div, double *copy) {
    const double inv = 1.0 / *d_div;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double x = v[i] * inv;
        v[i] = x;
        if (copy) copy[i] = x;
    }
}

VecArgs make_args(int64_t n, int K, const double *const *vecs, double *q, const double *w, ReduceScratch &rs,
                  double *d_out) {
    VecArgs a;
    a.n = n;
    a.K = K;
    for (int k = 0; k < kVecMaxK; ++k) {
        a.vec[k] = (vecs && k < K) ? vecs[k] : nullptr;
        a.c[k] = 0.0;
    }
    a.dc = nullptr;
    a.q = q;
    a.w = w;
    a.accumulate = false;
    a.d_out = d_out;
    a.partials = rs.partials;
    a.counter = rs.counter;
    return a;
}

int red_grid(int64_t n, const ReduceScratch &rs) {
    return stream_grid(n, 4, std::min(device_info().sm_count * 4, rs.max_ctas));
}

bool scratch_ok(const ReduceScratch &rs, int KP) { return rs.partials && rs.counter && rs.max_k >= KP; }

}  // namespace

cufsp_status vec_wdot(int64_t n, int K, const double *const *vecs, const double *q, const double *w, double *d_out,
                      ReduceScratch &rs, cudaStream_t st) {
    if (K < 1 || K > kVecMaxK) return set_error(CUFSP_ERR_INVALID_ARG, "vec_wdot: K out of range");
    const int KP = K <= 8 ? 8 : K <= 16 ? 16 : K <= 32 ? 32 : 64;
    if (!scratch_ok(rs, KP)) return set_error(CUFSP_ERR_INVALID_ARG, "vec_wdot: reduction scratch too small");
    VecArgs a = make_args(n, K, vecs, const_cast<double *>(q), w, rs, d_out);
    const int g = red_grid(n, rs);
    if (KP == 8) k_wdot<8><<<g, kRedThreads, 0, st>>>(a);
    else if (KP == 16) k_wdot<16><<<g, kRedThreads, 0, st>>>(a);
    else if (KP == 32) k_wdot<32><<<g, kRedThreads, 0, st>>>(a);
    else k_wdot<64><<<g, kRedThreads, 0, st>>>(a);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

cufsp_status vec_maxpy_wnorm(int64_t n, int K, const double *const *vecs, const double *d_c, double *q,
                             const double *w, double *d_norm, ReduceScratch &rs, cudaStream_t st) {
    if (K < 1 || K > kVecMaxK) return set_error(CUFSP_ERR_INVALID_ARG, "vec_maxpy_wnorm: K out of range");
    if (!scratch_ok(rs, 1)) return set_error(CUFSP_ERR_INVALID_ARG, "vec_maxpy_wnorm: no reduction scratch");
    VecArgs a = make_args(n, K, vecs, q, w, rs, d_norm);
    a.dc = d_c;
    const int g = red_grid(n, rs);
    if (K <= 8) k_maxpy_wnorm<8><<<g, kRedThreads, 0, st>>>(a);
    else if (K <= 16) k_maxpy_wnorm<16><<<g, kRedThreads, 0, st>>>(a);
    else if (K <= 32) k_maxpy_wnorm<32><<<g, kRedThreads, 0, st>>>(a);
    else k_maxpy_wnorm<64><<<g, kRedThreads, 0, st>>>(a);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

cufsp_status vec_lincomb(int64_t n, int K, const double *const *vecs, const double *c, double *out, bool accumulate,
                         const double *w, double *d_norm, ReduceScratch &rs, cudaStream_t st) {
    if (K < 1 || K > kVecMaxK) return set_error(CUFSP_ERR_INVALID_ARG, "vec_lincomb: K out of range");
    if (d_norm && !scratch_ok(rs, 1)) return set_error(CUFSP_ERR_INVALID_ARG, "vec_lincomb: no reduction scratch");
    VecArgs a = make_args(n, K, vecs, out, w, rs, d_norm);
    for (int k = 0; k < K; ++k) a.c[k] = c[k];
    a.accumulate = accumulate;
    const int g = d_norm ? red_grid(n, rs) : stream_grid(n, 4, device_info().sm_count * 8);
    if (K <= 8) k_lincomb<8><<<g, kRedThreads, 0, st>>>(a);
    else if (K <= 16) k_lincomb<16><<<g, kRedThreads, 0, st>>>(a);
    else if (K <= 32) k_lincomb<32><<<g, kRedThreads, 0, st>>>(a);
    else k_lincomb<64><<<g, kRedThreads, 0, st>>>(a);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

cufsp_status vec_normalize(int64_t n, double *v, const double *d_div, double *copy, cudaStream_t st) {
    k_normalize<<<stream_grid(n, 4, device_info().sm_count * 8), 256, 0, st>>>(n, v, d_div, copy);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

cufsp_status vec_wnorm(int64_t n, const double *x, const double *w, double *d_out, ReduceScratch &rs,
                       cudaStream_t st) {
    if (!scratch_ok(rs, 1)) return set_error(CUFSP_ERR_INVALID_ARG, "vec_wnorm: no reduction scratch");
    VecArgs a = make_args(n, 0, nullptr, const_cast<double *>(x), w, rs, d_out);
    k_wnorm<<<red_grid(n, rs), kRedThreads, 0, st>>>(a);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

}  // namespace cufsp
