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

// The exponential works on kp x kp matrices, kp = k rounded up to a multiple of 8, with A embedded
// as the leading block of block-diag(A, 0): exp of that is block-diag(exp A, I), so the padding
// changes nothing in the leading block and every column is a whole number of 8-double vectors.
// (GCC notes that a 64-byte vector changes the calling convention without AVX-512; the helpers below
// have internal linkage and are always inlined, so no call ever passes one.)
#pragma GCC diagnostic ignored "-Wpsabi"
typedef double v8 __attribute__((vector_size(64), aligned(8)));

__attribute__((always_inline)) inline v8 ld8(const double *p) {
    v8 v;
    std::memcpy(&v, p, sizeof(v));
    return v;
}
__attribute__((always_inline)) inline void st8(double *p, v8 v) { std::memcpy(p, &v, sizeof(v)); }

// C = A B, column-major kp x kp (kp % 8 == 0): four columns of C kept in vector registers while one
// column of A streams past.  Cloned for AVX-512, AVX2 and baseline x86-64; the loader picks the
// widest the host supports.
__attribute__((target_clones("avx512f", "avx2", "default"))) void matmul(int kp, const double *__restrict A,
                                                                         const double *__restrict B,
                                                                         double *__restrict C) {
    for (int j = 0; j < kp; j += 4) {
        const double *b0 = B + (size_t)j * kp, *b1 = b0 + kp, *b2 = b1 + kp, *b3 = b2 + kp;
        for (int r = 0; r < kp; r += 8) {
            v8 c0 = {0, 0, 0, 0, 0, 0, 0, 0}, c1 = c0, c2 = c0, c3 = c0;
            for (int l = 0; l < kp; ++l) {
                const v8 a = ld8(A + (size_t)l * kp + r);
                c0 += a * b0[l];
                c1 += a * b1[l];
                c2 += a * b2[l];
                c3 += a * b3[l];
            }
            st8(C + (size_t)j * kp + r, c0);
            st8(C + (size_t)(j + 1) * kp + r, c1);
            st8(C + (size_t)(j + 2) * kp + r, c2);
            st8(C + (size_t)(j + 3) * kp + r, c3);
        }
    }
}

// X = P^{-1} Q by LU with partial pivoting.  P and Q are column-major kp x kp on entry; they are
// transposed into row-major work arrays so that every elimination and substitution step is a
// contiguous row operation.  X (column-major) overwrites Q.  False if P is singular.
__attribute__((target_clones("avx512f", "avx2", "default"))) bool lu_solve(int kp, const double *__restrict Pc,
                                                                           double *__restrict Qc, double *__restrict P,
                                                                           double *__restrict Q) {
    for (int i = 0; i < kp; ++i)
        for (int j = 0; j < kp; ++j) {
            P[(size_t)i * kp + j] = Pc[i + (size_t)j * kp];
            Q[(size_t)i * kp + j] = Qc[i + (size_t)j * kp];
        }
    for (int c = 0; c < kp; ++c) {
        int p = c;
        double best = std::fabs(P[(size_t)c * kp + c]);
        for (int i = c + 1; i < kp; ++i) {
            const double v = std::fabs(P[(size_t)i * kp + c]);
            if (v > best) {
                best = v;
                p = i;
            }
        }
        if (best == 0.0) return false;
        if (p != c)
            for (int j = 0; j < kp; ++j) {
                std::swap(P[(size_t)c * kp + j], P[(size_t)p * kp + j]);
                std::swap(Q[(size_t)c * kp + j], Q[(size_t)p * kp + j]);
            }
        const double inv = 1.0 / P[(size_t)c * kp + c];
        const double *__restrict pc = P + (size_t)c * kp;
        const double *__restrict qc = Q + (size_t)c * kp;
        for (int i = c + 1; i < kp; ++i) {
            double *__restrict pi = P + (size_t)i * kp;
            double *__restrict qi = Q + (size_t)i * kp;
            const double l = pi[c] * inv;
            if (l == 0.0) continue;
            for (int j = c + 1; j < kp; ++j) pi[j] -= l * pc[j];
            for (int j = 0; j < kp; ++j) qi[j] -= l * qc[j];
        }
    }
    for (int c = kp - 1; c >= 0; --c) {  // back substitution, whole rows of Q at a time
        double *__restrict qc = Q + (size_t)c * kp;
        const double *__restrict pc = P + (size_t)c * kp;
        for (int i = c + 1; i < kp; ++i) {
            const double u = pc[i];
            if (u == 0.0) continue;
            const double *__restrict qi = Q + (size_t)i * kp;
            for (int j = 0; j < kp; ++j) qc[j] -= u * qi[j];
        }
        const double inv = 1.0 / pc[c];
        for (int j = 0; j < kp; ++j) qc[j] *= inv;
    }
    for (int i = 0; i < kp; ++i)
        for (int j = 0; j < kp; ++j) Qc[i + (size_t)j * kp] = Q[(size_t)i * kp + j];
    return true;
}

// C (m x n) = A (m x l) B (l x n), or C += A B when acc; column-major with leading dimensions, so
// that the blocks of a block-triangular matrix are multiplied in place.  m % 8 == 0, n % 4 == 0.
__attribute__((target_clones("avx512f", "avx2", "default"))) void matmul_rect(int m, int n, int l, const double *A,
                                                                              int lda, const double *B, int ldb,
                                                                              double *C, int ldc, bool acc) {
    for (int j = 0; j < n; j += 4) {
        const double *b0 = B + (size_t)j * ldb, *b1 = b0 + ldb, *b2 = b1 + ldb, *b3 = b2 + ldb;
        double *cj = C + (size_t)j * ldc;
        for (int r = 0; r < m; r += 8) {
            v8 c0 = {0, 0, 0, 0, 0, 0, 0, 0}, c1 = c0, c2 = c0, c3 = c0;
            if (acc) {
                c0 = ld8(cj + r);
                c1 = ld8(cj + ldc + r);
                c2 = ld8(cj + 2 * (size_t)ldc + r);
                c3 = ld8(cj + 3 * (size_t)ldc + r);
            }
            for (int q = 0; q < l; ++q) {
                const v8 a = ld8(A + (size_t)q * lda + r);
                c0 += a * b0[q];
                c1 += a * b1[q];
                c2 += a * b2[q];
                c3 += a * b3[q];
            }
            st8(cj + r, c0);
            st8(cj + ldc + r, c1);
            st8(cj + 2 * (size_t)ldc + r, c2);
            st8(cj + 3 * (size_t)ldc + r, c3);
        }
    }
}

// X = P^{-1} Q for P n x n and Q n x nrhs (column-major, leading dimensions ldp and ldq), by LU with
// partial pivoting on row-major copies (Pw: n x n, Qw: n x nrhs); X overwrites Q.  False if P is
// singular.
__attribute__((target_clones("avx512f", "avx2", "default"))) bool lu_solve_rect(int n, int nrhs, const double *Pc,
                                                                                int ldp, double *Qc, int ldq,
                                                                                double *__restrict P,
                                                                                double *__restrict Q) {
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) P[(size_t)i * n + j] = Pc[i + (size_t)j * ldp];
        for (int j = 0; j < nrhs; ++j) Q[(size_t)i * nrhs + j] = Qc[i + (size_t)j * ldq];
    }
    for (int c = 0; c < n; ++c) {
        int p = c;
        double best = std::fabs(P[(size_t)c * n + c]);
        for (int i = c + 1; i < n; ++i) {
            const double v = std::fabs(P[(size_t)i * n + c]);
            if (v > best) {
                best = v;
                p = i;
            }
        }
        if (best == 0.0) return false;
        if (p != c) {
            for (int j = 0; j < n; ++j) std::swap(P[(size_t)c * n + j], P[(size_t)p * n + j]);
            for (int j = 0; j < nrhs; ++j) std::swap(Q[(size_t)c * nrhs + j], Q[(size_t)p * nrhs + j]);
        }
        const double inv = 1.0 / P[(size_t)c * n + c];
        const double *__restrict pc = P + (size_t)c * n;
        const double *__restrict qc = Q + (size_t)c * nrhs;
        for (int i = c + 1; i < n; ++i) {
            double *__restrict pi = P + (size_t)i * n;
            double *__restrict qi = Q + (size_t)i * nrhs;
            const double l = pi[c] * inv;
            if (l == 0.0) continue;
            for (int j = c + 1; j < n; ++j) pi[j] -= l * pc[j];
            for (int j = 0; j < nrhs; ++j) qi[j] -= l * qc[j];
        }
    }
    for (int c = n - 1; c >= 0; --c) {
        double *__restrict qc = Q + (size_t)c * nrhs;
        const double *__restrict pc = P + (size_t)c * n;
        for (int i = c + 1; i < n; ++i) {
            const double u = pc[i];
            if (u == 0.0) continue;
            const double *__restrict qi = Q + (size_t)i * nrhs;
            for (int j = 0; j < nrhs; ++j) qc[j] -= u * qi[j];
        }
        const double inv = 1.0 / pc[c];
        for (int j = 0; j < nrhs; ++j) qc[j] *= inv;
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < nrhs; ++j) Qc[i + (size_t)j * ldq] = Q[(size_t)i * nrhs + j];
    return true;
}

// Block upper-triangular kp x kp matrices, kp = k1p + k2p: blocks X11 (k1p x k1p), X12 (k1p x k2p)
// and X22 (k2p x k2p) at their places in a column-major kp x kp array; the X21 block is kept zero.
struct BlockTri {
    int k1p, k2p, kp;
    double *b12(double *X) const { return X + (size_t)k1p * kp; }
    double *b22(double *X) const { return X + (size_t)k1p * kp + k1p; }
    const double *b12(const double *X) const { return X + (size_t)k1p * kp; }
    const double *b22(const double *X) const { return X + (size_t)k1p * kp + k1p; }
    void zero21(double *X) const {
        for (int j = 0; j < k1p; ++j) std::memset(X + (size_t)j * kp + k1p, 0, sizeof(double) * k2p);
    }
    // C = A B: three block products instead of the eight of a full product
    void mul(const double *A, const double *B, double *C) const {
        matmul_rect(k1p, k1p, k1p, A, kp, B, kp, C, kp, false);
        matmul_rect(k1p, k2p, k1p, A, kp, b12(B), kp, b12(C), kp, false);
        matmul_rect(k1p, k2p, k2p, b12(A), kp, b22(B), kp, b12(C), kp, true);
        matmul_rect(k2p, k2p, k2p, b22(A), kp, b22(B), kp, b22(C), kp, false);
        zero21(C);
    }
};

}  // namespace

cufsp_status expm_pade13(int k, const double *A, double *F) {
    if (k < 1 || !A || !F) return set_error(CUFSP_ERR_INVALID_ARG, "expm: bad argument");
    const int m = 13;
    double c[m + 1];
    c[0] = 1.0;
    for (int j = 0; j < m; ++j) c[j + 1] = c[j] * (double)(m - j) / ((double)(j + 1) * (double)(2 * m - j));

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

    const int kp = (k + 7) & ~7;
    const size_t sz = (size_t)kp * kp;
    thread_local std::vector<double> work;  // 12 kp x kp matrices, reused across calls
    if (work.size() < 12 * sz) work.assign(12 * sz, 0.0);
    double *B = work.data(), *B2 = B + sz, *B4 = B2 + sz, *B6 = B4 + sz, *T = B6 + sz, *U = T + sz, *V = U + sz,
           *W = V + sz, *P = W + sz, *Q = P + sz, *Pr = Q + sz, *Qr = Pr + sz;
    std::memset(B, 0, sizeof(double) * sz);
    for (int j = 0; j < k; ++j)
        for (int i = 0; i < k; ++i) B[i + (size_t)j * kp] = A[i + (size_t)j * k] * scale;
    matmul(kp, B, B, B2);
    matmul(kp, B2, B2, B4);
    matmul(kp, B4, B2, B6);
    // odd part U = B (B6 (c13 B6 + c11 B4 + c9 B2) + c7 B6 + c5 B4 + c3 B2 + c1 I)
    for (size_t i = 0; i < sz; ++i) T[i] = c[13] * B6[i] + c[11] * B4[i] + c[9] * B2[i];
    matmul(kp, B6, T, W);
    for (size_t i = 0; i < sz; ++i) W[i] += c[7] * B6[i] + c[5] * B4[i] + c[3] * B2[i];
    for (int i = 0; i < kp; ++i) W[i + (size_t)i * kp] += c[1];
    matmul(kp, B, W, U);
    // even part V = B6 (c12 B6 + c10 B4 + c8 B2) + c6 B6 + c4 B4 + c2 B2 + c0 I
    for (size_t i = 0; i < sz; ++i) T[i] = c[12] * B6[i] + c[10] * B4[i] + c[8] * B2[i];
    matmul(kp, B6, T, V);
    for (size_t i = 0; i < sz; ++i) V[i] += c[6] * B6[i] + c[4] * B4[i] + c[2] * B2[i];
    for (int i = 0; i < kp; ++i) V[i + (size_t)i * kp] += c[0];
    // (V - U) R = (V + U)
    for (size_t i = 0; i < sz; ++i) {
        P[i] = V[i] - U[i];
        Q[i] = V[i] + U[i];
    }
    if (!lu_solve(kp, P, Q, Pr, Qr)) return set_error(CUFSP_ERR_NONFINITE, "expm: singular Pade denominator");
    double *R = Q, *S = T;
    for (int i = 0; i < sq; ++i) {
        matmul(kp, R, R, S);
        std::swap(R, S);
    }
    for (int j = 0; j < k; ++j)
        for (int i = 0; i < k; ++i) F[i + (size_t)j * k] = R[i + (size_t)j * kp];
    for (size_t i = 0; i < (size_t)k * k; ++i)
        if (!std::isfinite(F[i])) return set_error(CUFSP_ERR_NONFINITE, "expm: result holds NaN/Inf");
    return CUFSP_SUCCESS;
}

// exp of a block upper-triangular matrix [[A11, A12], [0, A22]] (A11 k1 x k1, A22 k2 x k2; the
// lower-left block of A is not read), by the same scaling and squaring with Pade(13) as expm_pade13:
// every power, the two Pade polynomials and every squaring stay block upper-triangular, so a product
// costs three block products, and (V - U) R = (V + U) splits into R22 = P22^{-1} Q22 and
// [R11 R12] = P11^{-1} [Q11, Q12 - P12 R22].  The result equals the full algorithm's in exact
// arithmetic (the full LU never pivots across the zero block); F is the full (k1 + k2)^2 result,
// its lower-left block zero.  Each diagonal block is padded to a multiple of 8 as in expm_pade13.
cufsp_status expm_pade13_blocktri(int k1, int k2, const double *A, double *F) {
    if (k1 < 1 || k2 < 1 || !A || !F) return set_error(CUFSP_ERR_INVALID_ARG, "expm: bad argument");
    const int k = k1 + k2;
    const int m = 13;
    double c[m + 1];
    c[0] = 1.0;
    for (int j = 0; j < m; ++j) c[j + 1] = c[j] * (double)(m - j) / ((double)(j + 1) * (double)(2 * m - j));

    double norm1 = 0.0;  // 1-norm of the block-triangular matrix
    for (int j = 0; j < k; ++j) {
        double s = 0.0;
        for (int i = 0; i < (j < k1 ? k1 : k); ++i) s += std::fabs(A[i + (size_t)j * k]);
        norm1 = std::max(norm1, s);
    }
    if (!std::isfinite(norm1)) return set_error(CUFSP_ERR_NONFINITE, "expm: matrix holds NaN/Inf");
    const double theta13 = 5.371920351148152;
    int sq = 0;
    if (norm1 > theta13) sq = (int)std::ceil(std::log2(norm1 / theta13));
    const double scale = std::ldexp(1.0, -sq);

    BlockTri bt;
    bt.k1p = (k1 + 7) & ~7;
    bt.k2p = (k2 + 7) & ~7;
    bt.kp = bt.k1p + bt.k2p;
    const int kp = bt.kp, k1p = bt.k1p, k2p = bt.k2p;
    const size_t sz = (size_t)kp * kp;
    thread_local std::vector<double> work;  // 11 kp x kp matrices and the LU work, reused across calls
    const size_t lu_words = (size_t)k1p * k1p + (size_t)k1p * kp + (size_t)k2p * k2p + (size_t)k2p * k2p;
    if (work.size() < 11 * sz + lu_words) work.assign(11 * sz + lu_words, 0.0);
    double *B = work.data(), *B2 = B + sz, *B4 = B2 + sz, *B6 = B4 + sz, *T = B6 + sz, *U = T + sz, *V = U + sz,
           *W = V + sz, *P = W + sz, *Q = P + sz, *S = Q + sz, *lu = S + sz;
    std::memset(B, 0, sizeof(double) * sz);
    for (int j = 0; j < k; ++j) {  // A's blocks at their padded places
        const int jp = j < k1 ? j : j - k1 + k1p;
        for (int i = 0; i < (j < k1 ? k1 : k); ++i) {
            const int ip = i < k1 ? i : i - k1 + k1p;
            B[ip + (size_t)jp * kp] = A[i + (size_t)j * k] * scale;
        }
    }
    bt.mul(B, B, B2);
    bt.mul(B2, B2, B4);
    bt.mul(B4, B2, B6);
    // odd part U = B (B6 (c13 B6 + c11 B4 + c9 B2) + c7 B6 + c5 B4 + c3 B2 + c1 I)
    for (size_t i = 0; i < sz; ++i) T[i] = c[13] * B6[i] + c[11] * B4[i] + c[9] * B2[i];
    bt.mul(B6, T, W);
    for (size_t i = 0; i < sz; ++i) W[i] += c[7] * B6[i] + c[5] * B4[i] + c[3] * B2[i];
    for (int i = 0; i < kp; ++i) W[i + (size_t)i * kp] += c[1];
    bt.mul(B, W, U);
    // even part V = B6 (c12 B6 + c10 B4 + c8 B2) + c6 B6 + c4 B4 + c2 B2 + c0 I
    for (size_t i = 0; i < sz; ++i) T[i] = c[12] * B6[i] + c[10] * B4[i] + c[8] * B2[i];
    bt.mul(B6, T, V);
    for (size_t i = 0; i < sz; ++i) V[i] += c[6] * B6[i] + c[4] * B4[i] + c[2] * B2[i];
    for (int i = 0; i < kp; ++i) V[i + (size_t)i * kp] += c[0];
    for (size_t i = 0; i < sz; ++i) {
        P[i] = V[i] - U[i];
        Q[i] = V[i] + U[i];
    }
    // R22 = P22^{-1} Q22, then [R11 R12] = P11^{-1} [Q11, Q12 - P12 R22]; R overwrites Q
    double *lu_p1 = lu, *lu_q1 = lu_p1 + (size_t)k1p * k1p, *lu_p2 = lu_q1 + (size_t)k1p * kp,
           *lu_q2 = lu_p2 + (size_t)k2p * k2p;
    if (!lu_solve_rect(k2p, k2p, bt.b22(P), kp, bt.b22(Q), kp, lu_p2, lu_q2))
        return set_error(CUFSP_ERR_NONFINITE, "expm: singular Pade denominator");
    matmul_rect(k1p, k2p, k2p, bt.b12(P), kp, bt.b22(Q), kp, bt.b12(T), kp, false);  // Q12 -= P12 R22
    for (int j = 0; j < k2p; ++j)
        for (int i = 0; i < k1p; ++i) bt.b12(Q)[i + (size_t)j * kp] -= bt.b12(T)[i + (size_t)j * kp];
    if (!lu_solve_rect(k1p, kp, P, kp, Q, kp, lu_p1, lu_q1))  // Q11 and Q12 side by side: k1p x kp
        return set_error(CUFSP_ERR_NONFINITE, "expm: singular Pade denominator");
    bt.zero21(Q);
    double *R = Q;
    for (int i = 0; i < sq; ++i) {
        bt.mul(R, R, S);
        std::swap(R, S);
    }
    for (int j = 0; j < k; ++j) {
        const int jp = j < k1 ? j : j - k1 + k1p;
        for (int i = 0; i < k; ++i) {
            const int ip = i < k1 ? i : i - k1 + k1p;
            F[i + (size_t)j * k] = (i >= k1 && j < k1) ? 0.0 : R[ip + (size_t)jp * kp];
        }
    }
    for (size_t i = 0; i < (size_t)k * k; ++i)
        if (!std::isfinite(F[i])) return set_error(CUFSP_ERR_NONFINITE, "expm: result holds NaN/Inf");
    return CUFSP_SUCCESS;
}

}  // namespace cufsp

extern "C" cufsp_status cufsp_expm_host(int k, const double *A, double *F) { return cufsp::expm_pade13(k, A, F); }

extern "C" cufsp_status cufsp_expm_blocktri_host(int k1, int k2, const double *A, double *F) {
    return cufsp::expm_pade13_blocktri(k1, k2, A, F);
}
