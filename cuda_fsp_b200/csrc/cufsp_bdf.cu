// cufsp_bdf.cu -- variable-order BDF integrator for dp/dt = A(t) p on device vectors; replaces
// the SUNDIALS CVODE BDF + SPBCGS path that the reference drives through FSPMat::action
// (tests/test_sundials.cu:67-91, 142-200; problems/hog1p_5species.cu:203-228, 287-336).
//
// Method (published, not CVODE's code; SUNDIALS is not part of the reference):
//   * orders 1..5, quasi-constant step size in backward-difference form (Shampine & Reichelt,
//     SIAM J. Sci. Comput. 18(1), 1997), pure BDF coefficients alpha_k = gamma_k = sum 1/j,
//     local error constant 1/(k+1), step change by their matrix R(rho), order k-1/k/k+1 chosen
//     after k+1 equal steps;
//   * the CME is linear, so each step is one linear solve
//       (I - c A(t_new)) d = c A(t_new) y_pred - psi,   c = h / alpha_k,
//     by GMRES with classical Gram-Schmidt plus one re-orthogonalisation pass in the weighted
//     inner product <x, y>_w = sum x_i y_i w_i^2, w_i = 1 / ((atol + rtol |y_n,i|) sqrt(n)), so that
//     ||.||_w is the weighted RMS norm of the error test;
//   * starting step of Hairer, Norsett & Wanner (Solving ODEs I, Sec. II.4).
//
// Layout: the difference history D_0..D_7 (D_0 = y_n), the Krylov basis V_0..V_maxl and four work
// vectors live in one allocation with a row pitch rounded to 32 doubles (256 B) so that every
// vector is aligned for the vectorised generator kernels.  Every vector operation is one
// streaming kernel with a deterministic reduction; the host keeps the step-control scalars and
// reads back one small block per GMRES iteration.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cufsp_internal.h"
#include "cufsp_reduce.cuh"
#include "cufsp_vec.h"

using namespace cufsp;

namespace {

constexpr int kMaxOrder = 5;
constexpr int kNHist = kMaxOrder + 3;
constexpr int kMaxL = 60;

// device scalar block (doubles)
constexpr int kH1 = 0, kH2 = 64, kHN = 128, kBeta = 129, kErr = 130, kEm = 131, kEp = 132, kD0 = 133, kD1 = 134,
              kD2 = 135, kNScal = 136;

struct HistArgs {
    double *D[kNHist];
    int64_t n;
    int k;
};

// ypred = sum_{j<=k} D_j;   b = -(sum_{1<=j<=k} g_j D_j) / alpha
__global__ void __launch_bounds__(256) k_bdf_predict(const HistArgs h, double *ypred, double *b, double g1, double g2,
                                                     double g3, double g4, double g5, double inv_alpha) {
    const double g[kMaxOrder + 1] = {0.0, g1, g2, g3, g4, g5};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < h.n; i += stride) {
        double yp = 0.0, ps = 0.0;
#pragma unroll
        for (int j = 0; j <= kMaxOrder; ++j)
            if (j <= h.k) {
                const double dj = h.D[j][i];
                yp += dj;
                if (j >= 1) ps = fma(g[j], dj, ps);
            }
        ypred[i] = yp;
        b[i] = -ps * inv_alpha;
    }
}

struct MixArgs {
    double T[(kMaxOrder + 1) * (kMaxOrder + 1)];
};

// D_r <- sum_{j<=k} T[r][j] D_j,  r <= k
__global__ void __launch_bounds__(256) k_bdf_change(const HistArgs h, const MixArgs m) {
    const int k1 = h.k + 1;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < h.n; i += stride) {
        double old[kMaxOrder + 1];
#pragma unroll
        for (int j = 0; j <= kMaxOrder; ++j) old[j] = j < k1 ? h.D[j][i] : 0.0;
#pragma unroll
        for (int r = 0; r <= kMaxOrder; ++r) {
            if (r < k1) {
                double s = 0.0;
#pragma unroll
                for (int j = 0; j <= kMaxOrder; ++j)
                    if (j < k1) s += m.T[r * k1 + j] * old[j];
                h.D[r][i] = s;
            }
        }
    }
}

// Accepted step: D_{k+2} = d - D_{k+1}, D_{k+1} = d, D_j += D_{j+1} (j = k..0); new weights from
// y = D_0; out[0] = ||D_k||_w, out[1] = ||D_{k+2}||_w with the new weights.
__global__ void __launch_bounds__(kRedThreads) k_bdf_accept(const HistArgs h, const double *d, double *w, double atol,
                                                           double rtol, double sqrt_n, double *partials,
                                                           unsigned int *counter, double *out) {
    __shared__ RedSmem<2> sm;
    double acc[2] = {0.0, 0.0};
    const int k = h.k;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < h.n; i += stride) {
        double v[kNHist];
#pragma unroll
        for (int j = 0; j < kNHist; ++j) v[j] = (j <= k + 1) ? h.D[j][i] : 0.0;
        const double di = d[i];
        double top = 0.0;  // D_{k+2}
#pragma unroll
        for (int j = 0; j < kNHist; ++j)
            if (j == k + 1) {
                top = di - v[j];
                v[j] = di;
            }
#pragma unroll
        for (int j = kNHist - 2; j >= 0; --j)
            if (j <= k) v[j] += v[j + 1];
#pragma unroll
        for (int j = 0; j < kNHist; ++j)
            if (j <= k + 1) h.D[j][i] = v[j];
        if (k + 2 < kNHist) h.D[k + 2][i] = top;
        const double wi = 1.0 / ((atol + rtol * fabs(v[0])) * sqrt_n);
        w[i] = wi;
        double dk = 0.0;
#pragma unroll
        for (int j = 0; j < kNHist; ++j)
            if (j == k) dk = v[j];
        const double w2 = wi * wi;
        acc[0] = fma(dk * dk, w2, acc[0]);
        acc[1] = fma(top * top, w2, acc[1]);
    }
    if (grid_reduce<2>(acc, 2, partials, counter, sm) && threadIdx.x < 2) out[threadIdx.x] = sqrt(sm.final_[threadIdx.x]);
}

__global__ void __launch_bounds__(256) k_bdf_weights(int64_t n, const double *y, double *w, double atol, double rtol,
                                                     double sqrt_n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        w[i] = 1.0 / ((atol + rtol * fabs(y[i])) * sqrt_n);
}

// R(rho): R[0][j] = 1, R[i][0] = 0 (i > 0), R[i][j] = R[i-1][j] (i - 1 - rho j) / i
void bdf_R(int k, double rho, double R[kMaxOrder + 1][kMaxOrder + 1]) {
    for (int j = 0; j <= k; ++j) R[0][j] = 1.0;
    for (int i = 1; i <= k; ++i) {
        R[i][0] = 0.0;
        for (int j = 1; j <= k; ++j) R[i][j] = R[i - 1][j] * ((i - 1) - rho * j) / (double)i;
    }
}

}  // namespace

struct cufsp_bdf_s {
    cufsp_mat *A = nullptr;
    bool fixed = false;
    std::vector<double> coefs, cbuf;
    double rtol = 1e-8, atol = 1e-12, eps_lin = 0.005, h_init = 0.0, h_max = 0.0;
    int64_t max_steps = 1000000;
    int maxl = 30;
    int64_t n = 0, ld = 0;
    double *store = nullptr;
    double *D[kNHist] = {};
    double *V = nullptr;  // maxl + 1 vectors
    double *w = nullptr, *ypred = nullptr, *d = nullptr, *tmp = nullptr;
    double *d_scal = nullptr, *h_scal = nullptr;
    unsigned *h_seq = nullptr;  // sequence word of the scalar block (pinned host memory)
    unsigned seq = 0;
    ReduceScratch rs;
    double gam[kMaxOrder + 2] = {}, econst[kMaxOrder + 2] = {};
    // state
    bool ready = false, started = false;
    double t = 0.0, h = 0.0;
    int order = 1, n_equal = 0;
    cufsp_bdf_stats st{};

    double *vec(int j) const { return V + (int64_t)j * ld; }
};

namespace {

int grid_of(int64_t n) { return stream_grid(n, 4, device_info().sm_count * 8); }

HistArgs hist(const cufsp_bdf *B, int k) {
    HistArgs h;
    for (int j = 0; j < kNHist; ++j) h.D[j] = B->D[j];
    h.n = B->n;
    h.k = k;
    return h;
}

cufsp_status apply(cufsp_bdf *B, double t, double alpha, const double *x, bool accumulate, double *y,
                   cudaStream_t st) {
    cufsp_status s = mat_coefs(B->A, t, B->fixed ? B->coefs.data() : nullptr, B->cbuf);
    if (s != CUFSP_SUCCESS) return s;
    B->st.n_matvec++;
    return mat_apply(B->A, B->cbuf.data(), alpha, nullptr, nullptr, x, accumulate, y, st);
}

// Copies scalars [first, first + count) of the device block into the pinned host block (reachable
// from the device through unified addressing), then raises the sequence word.
__global__ void k_publish(const double *__restrict__ d, double *h, int first, int count, unsigned *h_seq,
                          unsigned seq) {
    if (threadIdx.x == 0) {
        for (int k = 0; k < count; ++k) h[first + k] = d[first + k];
        __threadfence_system();
        *(volatile unsigned *)h_seq = seq;
    }
}

bool spin_fetch() {  // CUFSP_BDF_SPIN=0: a copy command and a stream synchronisation instead
    static const bool on = [] {
        const char *e = getenv("CUFSP_BDF_SPIN");
        return !e || atoi(e) != 0;
    }();
    return on;
}

// The host reads the scalars the step control needs, once per GMRES iteration and a few times per
// step.  The scalars travel by k_publish and the host waits on the sequence word, which saves the copy
// command and the synchronisation call of each round trip.  The wait is bounded: the stream is
// queried every 1024 polls, and a finished or failed stream, or 10 s, ends it; a synchronisation then
// returns any error.
cufsp_status fetch(cufsp_bdf *B, int first, int count, cudaStream_t st) {
    if (!spin_fetch()) {
        CUFSP_CUDA_TRY(cudaMemcpyAsync(B->h_scal + first, B->d_scal + first, sizeof(double) * count,
                                       cudaMemcpyDeviceToHost, st));
        CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
        return mat_check_watchdog(B->A, "cufsp_bdf_advance");
    }
    const unsigned seq = ++B->seq;
    k_publish<<<1, 32, 0, st>>>(B->d_scal, B->h_scal, first, count, B->h_seq, seq);
    CUFSP_CUDA_TRY(cudaGetLastError());
    const auto t0 = std::chrono::steady_clock::now();
    for (unsigned it = 1; *(volatile unsigned *)B->h_seq != seq; ++it) {
        if ((it & 1023) == 0) {
            if (cudaStreamQuery(st) != cudaErrorNotReady) break;
            if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(10)) break;
        }
    }
    if (*(volatile unsigned *)B->h_seq != seq) CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
    return mat_check_watchdog(B->A, "cufsp_bdf_advance");
}

cufsp_status change_D(cufsp_bdf *B, int k, double rho, cudaStream_t st) {
    double R[kMaxOrder + 1][kMaxOrder + 1], U[kMaxOrder + 1][kMaxOrder + 1];
    bdf_R(k, rho, R);
    bdf_R(k, 1.0, U);
    MixArgs m;
    for (int i = 0; i <= k; ++i)
        for (int j = 0; j <= k; ++j) {
            double s = 0.0;  // (R U)[j][i]
            for (int l = 0; l <= k; ++l) s += R[j][l] * U[l][i];
            m.T[i * (k + 1) + j] = s;
        }
    k_bdf_change<<<grid_of(B->n), 256, 0, st>>>(hist(B, k), m);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

cufsp_status set_weights(cufsp_bdf *B, cudaStream_t st) {
    k_bdf_weights<<<grid_of(B->n), 256, 0, st>>>(B->n, B->D[0], B->w, B->atol, B->rtol, std::sqrt((double)B->n));
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

#define BDF_TRY(x)                                     \
    do {                                               \
        cufsp_status s_ = (x);                         \
        if (s_ != CUFSP_SUCCESS) return s_;            \
    } while (0)

// Starting step (Hairer, Norsett & Wanner) and D_1 = h f(t0, y0).
cufsp_status start(cufsp_bdf *B, double t_out, cudaStream_t st) {
    const int64_t n = B->n;
    double *f0 = B->tmp, *y1 = B->ypred, *f1 = B->d;
    BDF_TRY(apply(B, B->t, 1.0, B->D[0], false, f0, st));
    double h;
    if (B->h_init > 0.0) {
        h = B->h_init;
    } else {
        BDF_TRY(vec_wnorm(n, B->D[0], B->w, B->d_scal + kD0, B->rs, st));
        BDF_TRY(vec_wnorm(n, f0, B->w, B->d_scal + kD1, B->rs, st));
        BDF_TRY(fetch(B, kD0, 2, st));
        const double d0 = B->h_scal[kD0], d1 = B->h_scal[kD1];
        if (!std::isfinite(d0) || !std::isfinite(d1))
            return set_error(CUFSP_ERR_NONFINITE, "cufsp_bdf: initial vector or A(t0) p0 is not finite");
        double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
        h0 = std::min(h0, t_out - B->t);
        const double *v2[2] = {B->D[0], f0};
        const double c2[2] = {1.0, h0};
        BDF_TRY(vec_lincomb(n, 2, v2, c2, y1, false, nullptr, nullptr, B->rs, st));
        BDF_TRY(apply(B, B->t + h0, 1.0, y1, false, f1, st));
        const double *v3[2] = {f1, f0};
        const double c3[2] = {1.0 / h0, -1.0 / h0};
        BDF_TRY(vec_lincomb(n, 2, v3, c3, y1, false, B->w, B->d_scal + kD2, B->rs, st));
        BDF_TRY(fetch(B, kD2, 1, st));
        const double d2 = B->h_scal[kD2];
        const double h1 = (d1 <= 1e-15 && d2 <= 1e-15) ? std::max(1e-6, h0 * 1e-3) : std::sqrt(0.01 / std::max(d1, d2));
        h = std::min(100.0 * h0, h1);
    }
    const double hmax = B->h_max > 0.0 ? B->h_max : INFINITY;
    h = std::min(std::min(h, hmax), t_out - B->t);
    const double *v1[1] = {f0};
    BDF_TRY(vec_lincomb(n, 1, v1, &h, B->D[1], false, nullptr, nullptr, B->rs, st));
    B->h = h;
    B->started = true;
    return CUFSP_SUCCESS;
}

// GMRES on (I - c A(t)) d = b with b in V_0.  *conv = 1 when the residual reached eps_lin; then d
// holds the solution and d_scal[kErr] its weighted norm.
cufsp_status gmres(cufsp_bdf *B, double t, double c, cudaStream_t st, int *conv) {
    const int64_t n = B->n;
    *conv = 0;
    BDF_TRY(vec_wnorm(n, B->vec(0), B->w, B->d_scal + kBeta, B->rs, st));
    BDF_TRY(fetch(B, kBeta, 1, st));
    const double beta = B->h_scal[kBeta];
    if (!std::isfinite(beta)) return set_error(CUFSP_ERR_NONFINITE, "cufsp_bdf: right-hand side is not finite");
    if (beta <= B->eps_lin) {
        CUFSP_CUDA_TRY(cudaMemsetAsync(B->d, 0, sizeof(double) * n, st));
        CUFSP_CUDA_TRY(cudaMemsetAsync(B->d_scal + kErr, 0, sizeof(double), st));
        *conv = 1;
        return CUFSP_SUCCESS;
    }
    BDF_TRY(vec_normalize(n, B->vec(0), B->d_scal + kBeta, B->vec(1), st));
    double H[(kMaxL + 1) * kMaxL], g[kMaxL + 1], cs[kMaxL], sn[kMaxL], y[kMaxL];
    g[0] = beta;
    const double *vp[kVecMaxK];
    for (int j = 0; j <= B->maxl && j < kVecMaxK; ++j) vp[j] = B->vec(j);
    int J = 0;
    for (int j = 0; j < B->maxl; ++j) {
        double *q = B->vec(j + 1);
        // q = V_j - c A V_j  (q holds a copy of V_j)
        BDF_TRY(apply(B, t, -c, B->vec(j), true, q, st));
        B->st.n_lin_iters++;
        BDF_TRY(vec_wdot(n, j + 1, vp, q, B->w, B->d_scal + kH1, B->rs, st));
        BDF_TRY(vec_maxpy_wnorm(n, j + 1, vp, B->d_scal + kH1, q, B->w, B->d_scal + kHN, B->rs, st));
        BDF_TRY(vec_wdot(n, j + 1, vp, q, B->w, B->d_scal + kH2, B->rs, st));
        BDF_TRY(vec_maxpy_wnorm(n, j + 1, vp, B->d_scal + kH2, q, B->w, B->d_scal + kHN, B->rs, st));
        BDF_TRY(fetch(B, 0, kNScal, st));
        const double hn = B->h_scal[kHN];
        if (!std::isfinite(hn)) return set_error(CUFSP_ERR_NONFINITE, "cufsp_bdf: Krylov vector is not finite");
        double *col = H + (int64_t)j * (kMaxL + 1);
        for (int l = 0; l <= j; ++l) col[l] = B->h_scal[kH1 + l] + B->h_scal[kH2 + l];
        col[j + 1] = hn;
        for (int l = 0; l < j; ++l) {
            const double a = col[l], b = col[l + 1];
            col[l] = cs[l] * a + sn[l] * b;
            col[l + 1] = -sn[l] * a + cs[l] * b;
        }
        const double a = col[j], b = col[j + 1];
        const double r = std::hypot(a, b);
        cs[j] = r > 0.0 ? a / r : 1.0;
        sn[j] = r > 0.0 ? b / r : 0.0;
        col[j] = r;
        col[j + 1] = 0.0;
        g[j + 1] = -sn[j] * g[j];
        g[j] = cs[j] * g[j];
        J = j + 1;
        if (std::fabs(g[j + 1]) <= B->eps_lin || hn == 0.0) {
            *conv = 1;
            break;
        }
        if (j + 1 < B->maxl) BDF_TRY(vec_normalize(n, q, B->d_scal + kHN, B->vec(j + 2), st));
    }
    if (!*conv) return CUFSP_SUCCESS;
    for (int i = J - 1; i >= 0; --i) {
        double s = g[i];
        for (int l = i + 1; l < J; ++l) s -= H[(int64_t)l * (kMaxL + 1) + i] * y[l];
        y[i] = s / H[(int64_t)i * (kMaxL + 1) + i];
    }
    // d = V y, and ||d||_w for the local error test
    return vec_lincomb(n, J, vp, y, B->d, false, B->w, B->d_scal + kErr, B->rs, st);
}

// One attempt sequence ending in an accepted step toward t_out (never past it).
cufsp_status step(cufsp_bdf *B, double t_out, cudaStream_t st) {
    const int64_t n = B->n;
    const double eps = 2.220446049250313e-16;
    const double hmax = B->h_max > 0.0 ? B->h_max : INFINITY;
    for (;;) {
        if (B->h > hmax) {
            BDF_TRY(change_D(B, B->order, hmax / B->h, st));
            B->h = hmax;
            B->n_equal = 0;
        }
        bool landing = false;
        if (B->t + B->h >= t_out) {
            const double rho = (t_out - B->t) / B->h;
            if (rho != 1.0) BDF_TRY(change_D(B, B->order, rho, st));
            B->h = t_out - B->t;
            B->n_equal = 0;
            landing = true;
        }
        if (!(B->h > 4.0 * eps * std::fabs(B->t)))
            return set_error(CUFSP_ERR_STEP_LIMIT, "cufsp_bdf: step size underflow");
        const int k = B->order;
        const double t_new = landing ? t_out : B->t + B->h;
        const double alpha = B->gam[k], c = B->h / alpha;
        k_bdf_predict<<<grid_of(n), 256, 0, st>>>(hist(B, k), B->ypred, B->vec(0), B->gam[1], B->gam[2], B->gam[3],
                                                  B->gam[4], B->gam[5], 1.0 / alpha);
        CUFSP_CUDA_TRY(cudaGetLastError());
        BDF_TRY(apply(B, t_new, c, B->ypred, true, B->vec(0), st));
        int conv = 0;
        BDF_TRY(gmres(B, t_new, c, st, &conv));
        if (!conv) {
            B->st.n_lin_fail++;
            BDF_TRY(change_D(B, k, 0.5, st));
            B->h *= 0.5;
            B->n_equal = 0;
            continue;
        }
        BDF_TRY(fetch(B, kErr, 1, st));
        const double err = B->econst[k] * B->h_scal[kErr];
        if (!std::isfinite(err)) return set_error(CUFSP_ERR_NONFINITE, "cufsp_bdf: local error estimate is not finite");
        if (err > 1.0) {
            const double rho = std::max(0.2, 0.9 * std::pow(err, -1.0 / (k + 1)));
            BDF_TRY(change_D(B, k, rho, st));
            B->h *= rho;
            B->n_equal = 0;
            B->st.n_reject++;
            continue;
        }
        k_bdf_accept<<<stream_grid(n, 4, std::min(device_info().sm_count * 4, B->rs.max_ctas)), kRedThreads, 0, st>>>(
            hist(B, k), B->d, B->w, B->atol, B->rtol, std::sqrt((double)n), B->rs.partials, B->rs.counter,
            B->d_scal + kEm);
        CUFSP_CUDA_TRY(cudaGetLastError());
        B->t = t_new;
        B->st.n_steps++;
        B->n_equal++;
        B->st.last_err = err;
        if (B->n_equal >= k + 1) {
            BDF_TRY(fetch(B, kEm, 2, st));
            const double em = k > 1 ? B->econst[k - 1] * B->h_scal[kEm] : INFINITY;
            const double ep = k < kMaxOrder ? B->econst[k + 1] * B->h_scal[kEp] : INFINITY;
            const double fm = std::pow(em, -1.0 / k), f0 = std::pow(err, -1.0 / (k + 1)),
                         fp = std::pow(ep, -1.0 / (k + 2));
            int delta = 0;
            double best = f0;
            if (fm > best) {
                best = fm;
                delta = -1;
            }
            if (fp > best) {
                best = fp;
                delta = 1;
            }
            B->order = k + delta;
            const double rho = std::min(10.0, 0.9 * best);
            BDF_TRY(change_D(B, B->order, rho, st));
            B->h *= rho;
            B->n_equal = 0;
        }
        return CUFSP_SUCCESS;
    }
}

void release(cufsp_bdf *B) {
    if (B->store) cudaFree(B->store);
    if (B->d_scal) cudaFree(B->d_scal);
    if (B->h_scal) cudaFreeHost(B->h_scal);
    if (B->h_seq) cudaFreeHost(B->h_seq);
    B->store = B->d_scal = B->h_scal = nullptr;
    B->h_seq = nullptr;
    B->rs.release();
}

}  // namespace

extern "C" cufsp_status cufsp_bdf_create(cufsp_mat *A, const double *coefs, double rtol, double atol, int maxl,
                                         cufsp_bdf **out) {
    clear_error();
    if (!out || !A) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_create: NULL argument");
    *out = nullptr;
    if (!(rtol > 0.0) || !(atol > 0.0) || !std::isfinite(rtol) || !std::isfinite(atol))
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_create: rtol and atol must be finite and > 0");
    if (maxl < 1 || maxl > kMaxL) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_create: maxl must be 1..60");
    if (!coefs && !A->model.tcoef)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_create: no coefficients and the generator has no tcoef");
    cufsp_bdf *B = new cufsp_bdf();
    B->A = A;
    B->rtol = rtol;
    B->atol = atol;
    B->maxl = maxl;
    B->n = A->model.n;
    B->ld = (B->n + 31) / 32 * 32;
    if (coefs) {
        B->fixed = true;
        B->coefs.assign(coefs, coefs + A->model.nr);
    }
    B->gam[0] = 0.0;
    for (int k = 1; k <= kMaxOrder + 1; ++k) B->gam[k] = B->gam[k - 1] + 1.0 / k;
    for (int k = 0; k <= kMaxOrder + 1; ++k) B->econst[k] = 1.0 / (k + 1);
    const size_t nvec = kNHist + (size_t)(maxl + 1) + 4;
    cufsp_status s = CUFSP_SUCCESS;
    if (dev_malloc(&B->store, sizeof(double) * B->ld * nvec) != cudaSuccess ||
        dev_malloc(&B->d_scal, sizeof(double) * kNScal) != cudaSuccess ||
        cudaMallocHost(&B->h_scal, sizeof(double) * kNScal) != cudaSuccess ||
        cudaMallocHost(&B->h_seq, 64) != cudaSuccess) {
        cudaGetLastError();
        s = set_error(CUFSP_ERR_ALLOC, "cufsp_bdf_create: device allocation failed");
    }
    if (s == CUFSP_SUCCESS) *(volatile unsigned *)B->h_seq = 0u;
    if (s == CUFSP_SUCCESS) s = B->rs.init(device_info().sm_count * 4, 64);
    if (s != CUFSP_SUCCESS) {
        release(B);
        delete B;
        return s;
    }
    for (int j = 0; j < kNHist; ++j) B->D[j] = B->store + (int64_t)j * B->ld;
    B->V = B->store + (int64_t)kNHist * B->ld;
    double *work = B->V + (int64_t)(maxl + 1) * B->ld;
    B->w = work;
    B->ypred = work + B->ld;
    B->d = work + 2 * B->ld;
    B->tmp = work + 3 * B->ld;
    *out = B;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_bdf_destroy(cufsp_bdf *B) {
    if (!B) return CUFSP_SUCCESS;
    release(B);
    delete B;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_bdf_set_options(cufsp_bdf *B, double eps_lin, double h_init, double h_max,
                                              int64_t max_steps) {
    if (!B) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_set_options: NULL handle");
    if (!(eps_lin > 0.0) || !std::isfinite(eps_lin) || !std::isfinite(h_init) || !std::isfinite(h_max) ||
        max_steps < 1)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_set_options: bad option");
    B->eps_lin = eps_lin;
    B->h_init = h_init;
    B->h_max = h_max;
    B->max_steps = max_steps;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_bdf_set_coefs(cufsp_bdf *B, const double *coefs) {
    if (!B) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_set_coefs: NULL handle");
    if (!coefs && !B->A->model.tcoef)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_set_coefs: no coefficients and the generator has no tcoef");
    B->fixed = coefs != nullptr;
    if (coefs) B->coefs.assign(coefs, coefs + B->A->model.nr);
    B->ready = false;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_bdf_init(cufsp_bdf *B, double t0, const double *d_p0, cufsp_stream_t stream) {
    if (!B || !d_p0) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_init: NULL argument");
    if (!std::isfinite(t0)) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_init: t0 is not finite");
    cudaStream_t st = (cudaStream_t)stream;
    CUFSP_CUDA_TRY(cudaMemsetAsync(B->store, 0, sizeof(double) * B->ld * kNHist, st));
    CUFSP_CUDA_TRY(cudaMemcpyAsync(B->D[0], d_p0, sizeof(double) * B->n, cudaMemcpyDeviceToDevice, st));
    cufsp_status s = set_weights(B, st);
    if (s != CUFSP_SUCCESS) return s;
    B->t = t0;
    B->h = 0.0;
    B->order = 1;
    B->n_equal = 0;
    B->started = false;
    B->ready = true;
    std::memset(&B->st, 0, sizeof(B->st));
    B->st.t = t0;
    B->st.order = 1;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_bdf_advance(cufsp_bdf *B, double t_out, double *d_p, int one_step,
                                          cufsp_stream_t stream, double *t_reached) {
    if (!B || !d_p) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_advance: NULL argument");
    if (!B->ready) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_advance: call cufsp_bdf_init first");
    if (!std::isfinite(t_out) || t_out < B->t)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_advance: t_out must be finite and not before t");
    cudaStream_t st = (cudaStream_t)stream;
    const double eps = 2.220446049250313e-16;
    cufsp_status s = CUFSP_SUCCESS;
    if (!B->started && t_out > B->t) s = start(B, t_out, st);
    while (s == CUFSP_SUCCESS && B->t < t_out) {
        if (t_out - B->t <= 4.0 * eps * std::max(std::fabs(B->t), std::fabs(t_out))) {
            B->t = t_out;
            break;
        }
        if (B->st.n_steps >= B->max_steps) {
            s = set_error(CUFSP_ERR_STEP_LIMIT, "cufsp_bdf_advance: max_steps accepted steps did not reach t_out");
            break;
        }
        s = step(B, t_out, st);
        if (one_step) break;
    }
    B->st.t = B->t;
    B->st.h = B->h;
    B->st.order = B->order;
    if (s != CUFSP_SUCCESS) {
        B->ready = false;  // the history may be half-updated: a new init is required
        return s;
    }
    CUFSP_CUDA_TRY(cudaMemcpyAsync(d_p, B->D[0], sizeof(double) * B->n, cudaMemcpyDeviceToDevice, st));
    CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
    if (t_reached) *t_reached = B->t;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_bdf_get_stats(const cufsp_bdf *B, cufsp_bdf_stats *stats) {
    if (!B || !stats) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_bdf_get_stats: NULL argument");
    *stats = B->st;
    return CUFSP_SUCCESS;
}
