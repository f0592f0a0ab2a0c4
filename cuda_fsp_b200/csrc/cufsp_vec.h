// cufsp_vec.h -- multi-vector streaming primitives for the BDF integrator and its GMRES solver
// (cufsp_vec.cu).  Inner products are weighted, <x, y>_w = sum_i x_i y_i w_i^2, with w_i the
// error weights of the step (w = NULL: unweighted).  Reductions are deterministic.
#pragma once
#include "cufsp_internal.h"

namespace cufsp {

constexpr int kVecMaxK = 64;

// d_out[k] = <vecs[k], q>_w,  k < K <= 64
cufsp_status vec_wdot(int64_t n, int K, const double *const *vecs, const double *q, const double *w, double *d_out,
                      ReduceScratch &rs, cudaStream_t st);
// q -= sum_k d_c[k] vecs[k] (d_c on the device);  *d_norm = ||q||_w
cufsp_status vec_maxpy_wnorm(int64_t n, int K, const double *const *vecs, const double *d_c, double *q,
                             const double *w, double *d_norm, ReduceScratch &rs, cudaStream_t st);
// out = (accumulate ? out : 0) + sum_k c[k] vecs[k]  (c on the host); *d_norm = ||out||_w when d_norm
cufsp_status vec_lincomb(int64_t n, int K, const double *const *vecs, const double *c, double *out, bool accumulate,
                         const double *w, double *d_norm, ReduceScratch &rs, cudaStream_t st);
// v /= *d_div (device scalar);  copy = v when copy != NULL
cufsp_status vec_normalize(int64_t n, double *v, const double *d_div, double *copy, cudaStream_t st);
// *d_out = ||x||_w
cufsp_status vec_wnorm(int64_t n, const double *x, const double *w, double *d_out, ReduceScratch &rs,
                       cudaStream_t st);

}  // namespace cufsp
