// cufsp_expm.cpp -- dense matrix exponential for the small Krylov Hessenberg matrix.
//
// Replaces arma::expmat (called at src/KryExpvFSP.cu:125).  Method: scaling and squaring with
// the diagonal Pade(13,13) approximant (N. J. Higham, "The scaling and squaring method for the
// matrix exponential revisited", SIAM J. Matrix Anal. Appl. 26(4), 2005), degree 13 only:
//   s = max(0, ceil(log2(||A||_1 / theta_13))),  theta_13 = 5.371920351148152,
//   r13(B) = q(B)^{-1} p(B),  B = A / 2^s,  exp(A) = r13(B)^(2^s).
// The Pade coefficients are generated from c_0 = 1, c_{j+1} = c_j (m - j) / ((j + 1)(2m - j)),
// i.e. c_j = (2m-j)! m! / ((2m)! j! (m-j)!) with m = 13.  FP64 throughout, column-major.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "cufsp_internal.h"

namespace cufsp {

namespace {

// C = A * B, column-major, four columns of C per pass over A (the inner loop is unit-stride).
// Cloned for AVX-512, AVX2 and baseline x86-64; the loader picks the widest the host supports.
__attribute__((target_clones("avx512f", "avx2", "default"))) void matmul(int k, const double *__restrict A,
                                                                         const double *__restrict B,
                                                                         double *__restrict C) {
    int j = 0;
    for (; j + 4 <= k; j += 4) {
        double *__restrict c0 = C + (size_t)j * k;
        double *__restrict c1 = c0 + k;
        double *__restrict c2 = c1 + k;
        double *__restrict c3 = c2 + k;
        for (int i = 0; i < k; ++i) c0[i] = c1[i] = c2[i] = c3[i] = 0.0;
        for (int l = 0; l < k; ++l) {
            const double b0 = B[l + (size_t)j * k], b1 = B[l + (size_t)(j + 1) * k];
            const double b2 = B[l + (size_t)(j + 2) * k], b3 = B[l + (size_t)(j + 3) * k];
            const double *__restrict al = A + (size_t)l * k;
            for (int i = 0; i < k; ++i) {
                const double a = al[i];
                c0[i] += a * b0;
                c1[i] += a * b1;
                c2[i] += a * b2;
                c3[i] += a * b3;
            }
        }
    }
    for (; j < k; ++j) {
        double *__restrict cj = C + (size_t)j * k;
        for (int i = 0; i < k; ++i) cj[i] = 0.0;
        for (int l = 0; l < k; ++l) {
            const double b = B[l + (size_t)j * k];
            const double *__restrict al = A + (size_t)l * k;
            for (int i = 0; i < k; ++i) cj[i] += al[i] * b;
        }
    }
}

// Solve P X = Q in place (X overwrites Q) by LU with partial pivoting.  Returns false if P is
// singular to working precision.
bool lu_solve(int k, std::vector<double> &P, std::vector<double> &Q) {
    std::vector<int> piv(k);
    for (int c = 0; c < k; ++c) {
        int p = c;
        double best = std::fabs(P[c + (size_t)c * k]);
        for (int i = c + 1; i < k; ++i) {
            const double v = std::fabs(P[i + (size_t)c * k]);
            if (v > best) { best = v; p = i; }
        }
        if (best == 0.0) return false;
        piv[c] = p;
        if (p != c)
            for (int j = 0; j < k; ++j) std::swap(P[c + (size_t)j * k], P[p + (size_t)j * k]);
        const double inv = 1.0 / P[c + (size_t)c * k];
        for (int i = c + 1; i < k; ++i) P[i + (size_t)c * k] *= inv;
        for (int j = c + 1; j < k; ++j) {
            const double u = P[c + (size_t)j * k];
            if (u == 0.0) continue;
            for (int i = c + 1; i < k; ++i) P[i + (size_t)j * k] -= P[i + (size_t)c * k] * u;
        }
    }
    for (int j = 0; j < k; ++j) {
        double *q = Q.data() + (size_t)j * k;
        for (int c = 0; c < k; ++c)
            if (piv[c] != c) std::swap(q[c], q[piv[c]]);
        for (int c = 0; c < k; ++c)  // unit lower
            for (int i = c + 1; i < k; ++i) q[i] -= P[i + (size_t)c * k] * q[c];
        for (int c = k - 1; c >= 0; --c) {  // upper
            q[c] /= P[c + (size_t)c * k];
            for (int i = 0; i < c; ++i) q[i] -= P[i + (size_t)c * k] * q[c];
        }
    }
    return true;
}

}  // namespace

cufsp_status expm_pade13(int k, const double *A, double *F) {
    if (k < 1 || !A || !F) return set_error(CUFSP_ERR_INVALID_ARG, "expm: bad argument");
    const int m = 13;
    double c[m + 1];
    c[0] = 1.0;
    for (int j = 0; j < m; ++j) c[j + 1] = c[j] * (double)(m - j) / ((double)(j + 1) * (double)(2 * m - j));

    const size_t sz = (size_t)k * k;
    double norm1 = 0.0;
    for (int j = 0; j < k; ++j) {
        double s = 0.0;
        for (int i = 0; i < k; ++i) s += std::fabs(A[i + (size_t)j * k]);
        norm1 = std::max(norm1, s);
    }
    if (!std::isfinite(norm1)) return set_error(CUFSP_ERR_NONFINITE, "expm: matrix holds NaN/Inf");
    const double theta13 = 5.371920351148152;
    int sq = 0;
    if (norm1 > theta13) sq = (int)std::ceil(std::log2(norm1 / theta13));
    const double scale = std::ldexp(1.0, -sq);

    std::vector<double> B(sz), B2(sz), B4(sz), B6(sz), T(sz), U(sz), V(sz), W(sz);
    for (size_t i = 0; i < sz; ++i) B[i] = A[i] * scale;
    matmul(k, B.data(), B.data(), B2.data());
    matmul(k, B2.data(), B2.data(), B4.data());
    matmul(k, B4.data(), B2.data(), B6.data());
    // odd part U = B (B6 (c13 B6 + c11 B4 + c9 B2) + c7 B6 + c5 B4 + c3 B2 + c1 I)
    for (size_t i = 0; i < sz; ++i) T[i] = c[13] * B6[i] + c[11] * B4[i] + c[9] * B2[i];
    matmul(k, B6.data(), T.data(), W.data());
    for (size_t i = 0; i < sz; ++i) W[i] += c[7] * B6[i] + c[5] * B4[i] + c[3] * B2[i];
    for (int i = 0; i < k; ++i) W[i + (size_t)i * k] += c[1];
    matmul(k, B.data(), W.data(), U.data());
    // even part V = B6 (c12 B6 + c10 B4 + c8 B2) + c6 B6 + c4 B4 + c2 B2 + c0 I
    for (size_t i = 0; i < sz; ++i) T[i] = c[12] * B6[i] + c[10] * B4[i] + c[8] * B2[i];
    matmul(k, B6.data(), T.data(), V.data());
    for (size_t i = 0; i < sz; ++i) V[i] += c[6] * B6[i] + c[4] * B4[i] + c[2] * B2[i];
    for (int i = 0; i < k; ++i) V[i + (size_t)i * k] += c[0];
    // (V - U) R = (V + U)
    std::vector<double> P(sz), Q(sz);
    for (size_t i = 0; i < sz; ++i) {
        P[i] = V[i] - U[i];
        Q[i] = V[i] + U[i];
    }
    if (!lu_solve(k, P, Q)) return set_error(CUFSP_ERR_NONFINITE, "expm: singular Pade denominator");
    for (int i = 0; i < sq; ++i) {
        matmul(k, Q.data(), Q.data(), T.data());
        Q.swap(T);
    }
    std::memcpy(F, Q.data(), sizeof(double) * sz);
    for (size_t i = 0; i < sz; ++i)
        if (!std::isfinite(F[i])) return set_error(CUFSP_ERR_NONFINITE, "expm: result holds NaN/Inf");
    return CUFSP_SUCCESS;
}

}  // namespace cufsp

extern "C" cufsp_status cufsp_expm_host(int k, const double *A, double *F) { return cufsp::expm_pade13(k, A, F); }
