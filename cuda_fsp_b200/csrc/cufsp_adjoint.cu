// cufsp_adjoint.cu -- log-likelihood gradient by the adjoint method (no counterpart in the reference,
// whose Likelihood::evaluate, src/Likelihood.cpp:8-33, has no gradient).
//
//   log L(c) = sum_i sum_k D_i[k] log max(1e-44, q_i[k]),  q_i = M p(t_i),  p(t) = exp(t A(c)) p0,
//   A(c) = sum_r c_r A_r (A_r: reaction r at unit rate),  M sums each block of `block` states.
//
//   d log L / d c_r = int_0^T lambda(s)^T A_r p(s) ds,   lambda(T) = g_last,  lambda' = -A^T lambda,
//   lambda jumps by g_i = M^T (D_i / q_i) at each data time t_i (0 where q_i <= 1e-44).
//
// Forward pass: the adaptive Krylov solve (cufsp_krylov.cu) through the data times, storing p at
// every accepted step boundary (checkpoints) instead of the trajectory.  Backward pass, step by step
// in reverse: the forward Arnoldi basis V, H is rebuilt from the step's checkpoint (dense output
// p(s) = V exp((s - s0) H) beta e1 on the whole step); lambda is integrated backward over the step with
// the transposed generator (matrix-free A^T kernel) in adaptive sub-steps, each with its own basis U, G,
// lambda(s) = U exp((b - s) G) gamma e1.  On a sub-step [a, b] the integral is exact in the two
// subspaces:
//   int_a^b lambda^T A_r p ds = sum_{a', b'} W[a'][b'] u_{a'}^T A_r v_{b'},
//   W = int_0^tau exp((tau-u) G) z_b y_a^T exp(u H^T) du  = upper-right block of
//       exp(tau [[G, z_b y_a^T], [0, H^T]])   (Van Loan 1978),
// and the vector part is one fused kernel: uhat_{b'} = U W[:, b'] (multi-combination), then per state x
//   I_r += sum_{b'} v_{b'}(x) a_r(x) (uhat_{b'}(x + nu_r) 1{x + nu_r in box} - uhat_{b'}(x))
// for all reactions at once, with a deterministic grid reduction.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <string>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cufsp_internal.h"
#include "cufsp_reduce.cuh"

namespace cufsp {
namespace {

constexpr int kMaxB = CUFSP_MAX_KRYLOV + 1;

// g = M^T (D / q) for one data time: q[k] = sum of block k of p, g[x] = D[k] / q[k] (0 if q <= 1e-44).
__global__ void k_loglik_grad_vec(int64_t n, const double *__restrict__ p, int64_t block,
                                  const double *__restrict__ counts, double *__restrict__ g) {
    const int64_t nk = n / block;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += (int64_t)gridDim.x * blockDim.x) {
        double q = 0.0;
        for (int64_t j = 0; j < block; ++j) q += p[k * block + j];
        const double d = counts[k];
        const double v = (q > 1e-44 && d != 0.0) ? d / q : 0.0;
        for (int64_t j = 0; j < block; ++j) g[k * block + j] = v;
    }
}

__global__ void k_scale_vec(int64_t n, double a, double *__restrict__ x) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] *= a;
}

__global__ void k_axpy(int64_t n, double a, const double *__restrict__ x, double *__restrict__ y) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = fma(a, x[i], y[i]);
}

struct CombManyArgs {
    const double *in[kMaxB];
    double *out[kMaxB];
    int n_in, n_out;
    int64_t n;
    const double *coef;  // [n_in][n_out] (device)
};

// out_b = sum_a coef[a][b] in_a for all b, in one pass over the inputs: each thread keeps the NO
// output sums of its state in registers (same summation order as a loop over a per output).  The
// coefficient matrix is staged in shared memory with rows padded to NO and read as broadcast 16-byte
// pairs.  (Splitting the outputs over warp groups, 8 sums per thread at twice the occupancy, measured
// slower: 705 against 614 us on 2M states with 31 inputs and outputs.)
template <int NO>
__global__ void __launch_bounds__(256) k_comb_many(const CombManyArgs a) {
    __shared__ __align__(16) double cs[kMaxB * NO];
    for (int e = threadIdx.x; e < a.n_in * NO; e += blockDim.x) {
        const int ia = e / NO, b = e - ia * NO;
        cs[e] = b < a.n_out ? a.coef[ia * a.n_out + b] : 0.0;
    }
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc[NO];
#pragma unroll
        for (int k = 0; k < NO; ++k) acc[k] = 0.0;
#pragma unroll 2
        for (int ia = 0; ia < a.n_in; ++ia) {
            const double x = __ldg(a.in[ia] + i);
            const double2 *crow = reinterpret_cast<const double2 *>(cs + ia * NO);
#pragma unroll
            for (int k = 0; k < NO / 2; ++k) {
                const double2 c = crow[k];
                acc[2 * k] = fma(c.x, x, acc[2 * k]);
                acc[2 * k + 1] = fma(c.y, x, acc[2 * k + 1]);
            }
        }
#pragma unroll
        for (int k = 0; k < NO; ++k)
            if (k < a.n_out) a.out[k][i] = acc[k];
    }
}

void launch_comb_many(const CombManyArgs &ca, int grid, cudaStream_t st) {
    if (ca.n_out <= 8) k_comb_many<8><<<grid, 256, 0, st>>>(ca);
    else if (ca.n_out <= 16) k_comb_many<16><<<grid, 256, 0, st>>>(ca);
    else if (ca.n_out <= 32) k_comb_many<32><<<grid, 256, 0, st>>>(ca);
    else k_comb_many<64><<<grid, 256, 0, st>>>(ca);
}

struct BilinArgs {
    const double *v[kMaxB];     // forward basis W_b (scaled by vscale[b])
    const double *uh[kMaxB];    // uhat_b
    double vscale[kMaxB];
    int nb;
    const double *tables;
    const int *nu;              // [nr][ns] (device)
    int n, ns, nr, tab_stride;
    int dims[CUFSP_MAX_SPECIES];
    int tab_off[CUFSP_MAX_SPECIES];
    FastDiv div[CUFSP_MAX_SPECIES];
    int delta[CUFSP_MAX_REACTIONS];
    double *acc_out;            // [nr] accumulated (+=) by the last CTA
    double *partials;
    unsigned int *counter;
};

// I_r += sum_x a_r(x) sum_b v_b(x) (uhat_b(x + nu_r) 1{in box} - uhat_b(x))  for every r at once.
// Per state: the factors a_r(x) and target indices of all reactions first (NR >= nr, unrolled), then
// one pass over the basis: v_b(x) is read once and multiplies uhat_b at the state and at every
// reaction's target.  Same summation order per reaction as a loop over b per reaction.
template <int NR>
__global__ void __launch_bounds__(kRedThreads) k_adj_bilinear(const BilinArgs a) {
    __shared__ RedSmem<32> sm;
    double acc[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) acc[r] = 0.0;
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        int xs[CUFSP_MAX_SPECIES];
        unsigned rem = (unsigned)i;
        for (int s = 0; s < a.ns - 1; ++s) {
            const unsigned q = fd_div(rem, a.div[s]);
            xs[s] = (int)(rem - q * (unsigned)a.dims[s]);
            rem = q;
        }
        xs[a.ns - 1] = (int)rem;
        double f[NR];
        int j[NR];
        bool ok[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            f[r] = 0.0;
            ok[r] = false;
            j[r] = i;
            if (r < a.nr) {
                double fr = 1.0;
                bool okr = true;
                const double *tr = a.tables + (size_t)r * a.tab_stride;
                for (int s = 0; s < a.ns; ++s) {
                    fr *= __ldg(tr + a.tab_off[s] + xs[s]);
                    const int t = xs[s] + __ldg(a.nu + r * a.ns + s);
                    okr = okr && t >= 0 && t < a.dims[s];
                }
                f[r] = fr;
                ok[r] = okr;
                if (okr) j[r] = i + a.delta[r];
            }
        }
        double dsum = 0.0, os[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) os[r] = 0.0;
        for (int b = 0; b < a.nb; ++b) {
            const double wb = a.vscale[b] * __ldg(a.v[b] + i);
            const double *u = a.uh[b];
            dsum = fma(wb, __ldg(u + i), dsum);
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (ok[r]) os[r] = fma(wb, __ldg(u + j[r]), os[r]);
        }
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] += f[r] * ((ok[r] ? os[r] : 0.0) - dsum);
    }
    if (!grid_reduce<32>(acc, a.nr, a.partials, a.counter, sm)) return;
    for (int r = threadIdx.x; r < a.nr; r += blockDim.x) a.acc_out[r] += sm.final_[r];
}

void launch_adj_bilinear(const BilinArgs &ba, int grid, cudaStream_t st) {
    if (ba.nr <= 4) k_adj_bilinear<4><<<grid, kRedThreads, 0, st>>>(ba);
    else if (ba.nr <= 8) k_adj_bilinear<8><<<grid, kRedThreads, 0, st>>>(ba);
    else if (ba.nr <= 12) k_adj_bilinear<12><<<grid, kRedThreads, 0, st>>>(ba);
    else if (ba.nr <= 16) k_adj_bilinear<16><<<grid, kRedThreads, 0, st>>>(ba);
    else if (ba.nr <= 24) k_adj_bilinear<24><<<grid, kRedThreads, 0, st>>>(ba);
    else k_adj_bilinear<32><<<grid, kRedThreads, 0, st>>>(ba);
}

// beta * exp(s H) e1 for an mb x mb column-major H (host).
cufsp_status dense_output(int mb, const std::vector<double> &H, double s, double beta, std::vector<double> &y) {
    y.assign(mb, 0.0);
    if (mb == 0) return CUFSP_SUCCESS;
    std::vector<double> X((size_t)mb * mb), F((size_t)mb * mb);
    for (size_t i = 0; i < X.size(); ++i) X[i] = s * H[i];
    cufsp_status st = expm_pade13(mb, X.data(), F.data());
    if (st != CUFSP_SUCCESS) return st;
    for (int i = 0; i < mb; ++i) y[i] = beta * F[i];
    return CUFSP_SUCCESS;
}

struct Checkpoint {
    double *p;
    double tau;
};

// Work buffers of one gradient, from the buffer cache; all their uses are ordered on `st`, so their
// release waits for nothing on other streams (a concurrent gradient on another stream keeps running).
struct AdjWork {
    cudaStream_t st;
    std::vector<double *> bufs;
    explicit AdjWork(cudaStream_t s) : st(s) {}
    ~AdjWork() {
        for (double *b : bufs) cache_free(b, st);
    }
    double *alloc(size_t n) {
        double *p = nullptr;
        if (cache_alloc((void **)&p, sizeof(double) * n) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        bufs.push_back(p);
        return p;
    }
};

struct ExpvGuard {
    cufsp_expv *E = nullptr;
    ~ExpvGuard() {
        if (E) cufsp_expv_destroy(E);
    }
};

}  // namespace
}  // namespace cufsp

using namespace cufsp;

extern "C" cufsp_status cufsp_likelihood_grad(cufsp_mat *A, const double *coefs, int n_times, const double *times,
                                              const double *d_p0, int64_t block, const double *d_counts, int m,
                                              double tol, double *logL, double *grad, cufsp_stream_t stream) {
    clear_error();
    if (!A || !coefs || !times || !d_p0 || !d_counts || !logL || !grad || n_times < 1)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_likelihood_grad: NULL argument");
    if (!A->kron) return set_error(CUFSP_ERR_UNSUPPORTED, "cufsp_likelihood_grad: needs a KRONECKER generator");
    const int64_t n = A->model.n;
    const int nr = A->model.nr, ns = A->model.ns;
    if (block < 1 || n % block != 0) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_likelihood_grad: bad block");
    if (nr > 32) return set_error(CUFSP_ERR_UNSUPPORTED, "cufsp_likelihood_grad: at most 32 reactions");
    for (int i = 0; i < n_times; ++i)
        if (!(times[i] >= (i ? times[i - 1] : 0.0)) || !std::isfinite(times[i]))
            return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_likelihood_grad: times must be finite and non-decreasing");
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<double> c(coefs, coefs + nr);
    for (double v : c)
        if (!std::isfinite(v)) return set_error(CUFSP_ERR_NONFINITE, "cufsp_likelihood_grad: coefficient is NaN/Inf");

    ExpvGuard ef, eb;
    cufsp_status s = cufsp_expv_create(n, m, tol, 0, 2, 1.0, &ef.E);
    if (s == CUFSP_SUCCESS) s = cufsp_expv_create(n, m, tol, 0, 2, 1.0, &eb.E);
    if (s == CUFSP_SUCCESS) s = cufsp_expv_bind_mat_coefs(ef.E, A, c.data());
    if (s == CUFSP_SUCCESS) s = cufsp_expv_bind_mat_coefs(eb.E, A, c.data());
    if (s != CUFSP_SUCCESS) return s;
    expv_set_transpose(eb.E, true);

    AdjWork wk(st);
    double *p = wk.alloc(n), *lam = wk.alloc(n), *lam_b = wk.alloc(n), *pf = wk.alloc(n);
    double *g = wk.alloc((size_t)n * n_times);
    double *uh = wk.alloc((size_t)n * (m + 1));
    double *d_misc = wk.alloc(64 + (size_t)kMaxB * kMaxB);  // [0..31] I_r, [32] loglik, [64..] coefficient matrix
    ReduceScratch rs;
    if (!p || !lam || !lam_b || !pf || !g || !uh || !d_misc)
        return set_error(CUFSP_ERR_ALLOC, "cufsp_likelihood_grad: device allocation failed");
    struct RsGuard {
        ReduceScratch &r;
        cudaStream_t st;
        ~RsGuard() { r.release(st); }
    } rsg{rs, st};
    const int red_grid = stream_grid(n, 4, device_info().sm_count * 4);
    s = rs.init(red_grid, 32, st);
    if (s != CUFSP_SUCCESS) return s;
    double *d_I = d_misc, *d_ll = d_misc + 32, *d_coef = d_misc + 64;
    CUFSP_CUDA_TRY(cudaMemsetAsync(d_misc, 0, sizeof(double) * 64, st));
    const int vgrid = stream_grid(n, 4, device_info().sm_count * 8);

    // ---- forward pass with checkpoints ----
    CUFSP_CUDA_TRY(cudaMemcpyAsync(p, d_p0, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    std::vector<std::vector<Checkpoint>> steps(n_times);
    double *ck_next = nullptr;
    int ck_left = 0;
    // optional phase timers (CUFSP_VERBOSE=1)
    const bool verbose = getenv("CUFSP_VERBOSE") && atoi(getenv("CUFSP_VERBOSE")) != 0;
    using clk = std::chrono::steady_clock;
    double t_fwd = 0, t_arn = 0, t_bstep = 0, t_vl = 0, t_kern = 0;
    int n_sub = 0;
    auto since = [](clk::time_point a) { return std::chrono::duration<double>(clk::now() - a).count(); };
    const clk::time_point t_start = clk::now();
    double ll = 0.0, t_prev = 0.0;
    for (int i = 0; i < n_times; ++i) {
        const double dt = times[i] - t_prev;
        t_prev = times[i];
        if (dt > 0.0) {
            CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
            s = cufsp_expv_set_final_time(ef.E, dt);
            if (s == CUFSP_SUCCESS) s = cufsp_expv_reset_time(ef.E);
            if (s != CUFSP_SUCCESS) return s;
            int reached = 0;
            while (!reached) {
                if (ck_left == 0) {  // checkpoints are allocated 16 vectors at a time
                    ck_next = wk.alloc((size_t)n * 16);
                    if (!ck_next) return set_error(CUFSP_ERR_ALLOC, "cufsp_likelihood_grad: checkpoint allocation failed");
                    ck_left = 16;
                }
                double *ck = ck_next;
                ck_next += n;
                --ck_left;
                CUFSP_CUDA_TRY(cudaMemcpyAsync(ck, p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
                s = expv_step_once(ef.E, p, st);
                if (s != CUFSP_SUCCESS) return s;
                steps[i].push_back({ck, expv_last(ef.E).tau});
                cufsp_expv_final_time_reached(ef.E, &reached);
            }
        }
        double li = 0.0;
        s = cufsp_loglik(n, p, block, d_counts + (size_t)i * (n / block), &li, stream);
        if (s != CUFSP_SUCCESS) return s;
        ll += li;
        k_loglik_grad_vec<<<vgrid, 256, 0, st>>>(n, p, block, d_counts + (size_t)i * (n / block), g + (size_t)i * n);
        CUFSP_CUDA_TRY(cudaGetLastError());
    }

    // ---- backward pass ----
    CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
    t_fwd = since(t_start);
    CUFSP_CUDA_TRY(cudaMemsetAsync(lam, 0, sizeof(double) * n, st));
    BilinArgs ba;
    std::memset(&ba, 0, sizeof(ba));
    ba.tables = nullptr;
    const ModelHost &mh = A->model;
    // device copies of the model tables / stoichiometry for the bilinear kernel
    double *d_tab = wk.alloc(mh.tables.size());
    double *d_nu_d = wk.alloc((mh.nu.size() + 1) / 2 + 1);  // int storage inside a double buffer
    if (!d_tab || !d_nu_d) return set_error(CUFSP_ERR_ALLOC, "cufsp_likelihood_grad: device allocation failed");
    CUFSP_CUDA_TRY(cudaMemcpyAsync(d_tab, mh.tables.data(), sizeof(double) * mh.tables.size(), cudaMemcpyHostToDevice, st));
    CUFSP_CUDA_TRY(cudaMemcpyAsync(d_nu_d, mh.nu.data(), sizeof(int) * mh.nu.size(), cudaMemcpyHostToDevice, st));
    ba.tables = d_tab;
    ba.nu = reinterpret_cast<const int *>(d_nu_d);
    ba.n = (int)n;
    ba.ns = ns;
    ba.nr = nr;
    ba.tab_stride = mh.tab_stride;
    {
        int64_t stride = 1;
        for (int sp = 0; sp < ns; ++sp) {
            ba.dims[sp] = mh.bounds[sp] + 1;
            ba.tab_off[sp] = mh.tab_off[sp];
            ba.div[sp] = make_fastdiv((uint32_t)ba.dims[sp]);
            stride *= ba.dims[sp];
        }
        for (int r = 0; r < nr; ++r) {
            int64_t d = 0, stv = 1;
            for (int sp = 0; sp < ns; ++sp) {
                d += (int64_t)mh.nu[(size_t)r * ns + sp] * stv;
                stv *= ba.dims[sp];
            }
            ba.delta[r] = (int)std::max<int64_t>(-n, std::min<int64_t>(n, d));
        }
    }
    ba.acc_out = d_I;
    ba.partials = rs.partials;
    ba.counter = rs.counter;

    std::vector<double> ya, Xb, Fb, coefm;
    for (int i = n_times - 1; i >= 0; --i) {
        k_axpy<<<vgrid, 256, 0, st>>>(n, 1.0, g + (size_t)i * n, lam);
        CUFSP_CUDA_TRY(cudaGetLastError());
        double s_end = times[i];  // end of the current forward step
        for (int k = (int)steps[i].size() - 1; k >= 0; --k) {
            const Checkpoint &ck = steps[i][k];
            const double h = ck.tau;
            const double s0 = s_end - h;
            // forward basis on this step from its checkpoint
            clk::time_point tp = clk::now();
            CUFSP_CUDA_TRY(cudaMemcpyAsync(pf, ck.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
            s = expv_arnoldi(ef.E, pf, st);
            if (s != CUFSP_SUCCESS) return s;
            t_arn += since(tp);
            const KrylovStep F = expv_last(ef.E);
            // lambda backward over [s0, s_end] in adaptive sub-steps.  Expokit's error test is
            // absolute while |lambda| grows with the counts (g = D / q), so lambda is scaled to unit
            // norm for the solve and the step integrals are scaled back.
            s = launch_nrm2(n, lam, d_ll, rs, st);
            if (s != CUFSP_SUCCESS) return s;
            double lnorm = 0.0;
            CUFSP_CUDA_TRY(cudaMemcpyAsync(&lnorm, d_ll, sizeof(double), cudaMemcpyDeviceToHost, st));
            CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
            const double lscale = (lnorm > 0.0 && std::isfinite(lnorm)) ? lnorm : 1.0;
            k_scale_vec<<<vgrid, 256, 0, st>>>(n, 1.0 / lscale, lam);
            CUFSP_CUDA_TRY(cudaGetLastError());
            s = cufsp_expv_set_final_time(eb.E, h);
            if (s == CUFSP_SUCCESS) s = cufsp_expv_reset_time(eb.E);
            if (s != CUFSP_SUCCESS) return s;
            double b_end = s_end;
            int reached = h <= 0.0;
            while (!reached) {
                tp = clk::now();
                CUFSP_CUDA_TRY(cudaMemcpyAsync(lam_b, lam, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
                s = expv_step_once(eb.E, lam, st);
                if (s != CUFSP_SUCCESS) return s;
                t_bstep += since(tp);
                ++n_sub;
                const KrylovStep B = expv_last(eb.E);
                cufsp_expv_final_time_reached(eb.E, &reached);
                const double tau = B.tau;
                const double a0 = b_end - tau;
                if (F.beta > 0.0 && B.beta > 0.0 && tau > 0.0) {
                    tp = clk::now();
                    // W = upper-right mb_b x mb_f block of exp(tau [[G, z_b y_a^T], [0, H^T]])
                    s = dense_output(F.mb, F.H, a0 - s0, F.beta, ya);
                    if (s != CUFSP_SUCCESS) return s;
                    const int mbb = B.mb, mbf = F.mb, K = mbb + mbf;
                    Xb.assign((size_t)K * K, 0.0);
                    Fb.assign((size_t)K * K, 0.0);
                    for (int jj = 0; jj < mbb; ++jj)
                        for (int ii = 0; ii < mbb; ++ii) Xb[ii + (size_t)jj * K] = tau * B.H[ii + (size_t)jj * mbb];
                    for (int jj = 0; jj < mbf; ++jj) Xb[0 + (size_t)(mbb + jj) * K] = tau * B.beta * ya[jj];
                    for (int jj = 0; jj < mbf; ++jj)
                        for (int ii = 0; ii < mbf; ++ii)
                            Xb[(mbb + ii) + (size_t)(mbb + jj) * K] = tau * F.H[jj + (size_t)ii * mbf];  // H^T
                    s = expm_pade13_blocktri(mbb, mbf, Xb.data(), Fb.data());
                    if (s != CUFSP_SUCCESS) return s;
                    // uhat_b = sum_a W[a][b] rho_b[a] Ub_a
                    coefm.assign((size_t)mbb * mbf, 0.0);
                    for (int aa = 0; aa < mbb; ++aa)
                        for (int bb = 0; bb < mbf; ++bb)
                            coefm[(size_t)aa * mbf + bb] = lscale * Fb[aa + (size_t)(mbb + bb) * K] * B.rho[aa];
                    t_vl += since(tp);
                    tp = clk::now();
                    CUFSP_CUDA_TRY(cudaMemcpyAsync(d_coef, coefm.data(), sizeof(double) * coefm.size(),
                                                   cudaMemcpyHostToDevice, st));
                    CombManyArgs ca;
                    ca.n_in = mbb;
                    ca.n_out = mbf;
                    ca.n = n;
                    ca.coef = d_coef;
                    for (int aa = 0; aa < mbb; ++aa) ca.in[aa] = expv_basis(eb.E, lam_b, aa);
                    for (int bb = 0; bb < mbf; ++bb) ca.out[bb] = uh + (size_t)bb * n;
                    launch_comb_many(ca, vgrid, st);
                    CUFSP_CUDA_TRY(cudaGetLastError());
                    ba.nb = mbf;
                    for (int bb = 0; bb < mbf; ++bb) {
                        ba.v[bb] = expv_basis(ef.E, pf, bb);
                        ba.vscale[bb] = F.rho[bb];
                        ba.uh[bb] = uh + (size_t)bb * n;
                    }
                    launch_adj_bilinear(ba, red_grid, st);
                    CUFSP_CUDA_TRY(cudaGetLastError());
                    // No synchronisation: d_coef, uh and the bases are reused in stream order, and the
                    // pageable copy above has taken coefm before returning.  (With CUFSP_VERBOSE the
                    // kernels' time then shows in the next sub-step's "backward steps" phase.)
                    t_kern += since(tp);
                }
                b_end = a0;
            }
            k_scale_vec<<<vgrid, 256, 0, st>>>(n, lscale, lam);
            CUFSP_CUDA_TRY(cudaGetLastError());
            s_end = s0;
        }
    }
    std::vector<double> I(nr);
    CUFSP_CUDA_TRY(cudaMemcpyAsync(I.data(), d_I, sizeof(double) * nr, cudaMemcpyDeviceToHost, st));
    CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
    (void)d_ll;
    if (verbose) {
        size_t nsteps = 0;
        for (auto &v : steps) nsteps += v.size();
        fprintf(stderr,
                "cufsp_likelihood_grad: %zu forward steps, %d backward sub-steps; forward %.3f s, basis rebuild "
                "%.3f s, backward steps %.3f s, Van Loan %.3f s, step integrals %.3f s, total %.3f s\n",
                nsteps, n_sub, t_fwd, t_arn, t_bstep, t_vl, t_kern, since(t_start));
    }
    *logL = ll;
    for (int r = 0; r < nr; ++r) grad[r] = c[r] * I[r];  // d log L / d log c_r
    return CUFSP_SUCCESS;
}

// Many parameter sets: `workers` host threads, each with its own generator (the plane kernel keeps
// coefficient-dependent tables per generator), stream and Krylov workspaces, take sets from a shared
// counter; their solves overlap on the GPU.
extern "C" cufsp_status cufsp_likelihood_grad_batched(const cufsp_model_desc *desc, int n_sets, const double *coefs,
                                                      int n_times, const double *times, const double *d_p0,
                                                      int64_t block, const double *d_counts, int m, double tol,
                                                      int workers, double *logL, double *grad) {
    clear_error();
    if (!desc || !desc->fsp_bounds || desc->n_species < 1 || desc->n_species > CUFSP_MAX_SPECIES || !coefs || !logL ||
        !grad || n_sets < 1)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_likelihood_grad_batched: bad argument");
    const int nr = desc->n_reactions;
    workers = std::max(1, std::min(std::min(workers, n_sets), 32));
    // Generators small enough for the persistent Arnoldi pass: every worker's passes take an equal
    // share of the SMs (CUFSP_GRAD_SM_SHARE=0: each pass takes all SMs and the passes of the workers
    // take turns), so that the workers' solves run side by side; larger generators run `workers`
    // concurrent launch sequences.
    int64_t n_states = 1;
    for (int s = 0; s < desc->n_species; ++s) n_states *= (int64_t)desc->fsp_bounds[s] + 1;
    const bool persistent = parnoldi_size_ok(n_states);
    const char *share_env = getenv("CUFSP_GRAD_SM_SHARE");
    const bool share = !share_env || atoi(share_env) != 0;
    int cta_cap = 0;
    if (persistent && share) cta_cap = std::max(1, device_info().sm_count / workers);
    else if (persistent) workers = std::min(workers, 2);
    int dev = 0;
    CUFSP_CUDA_TRY(cudaGetDevice(&dev));
    // the workers' streams do not wait for the legacy default stream, where the caller's copies of
    // p0 and the counts were most likely queued
    CUFSP_CUDA_TRY(upload_fence());
    std::atomic<int> next(0);
    std::vector<cufsp_status> status(workers, CUFSP_SUCCESS);
    std::vector<std::string> msg(workers);
    auto work = [&](int w) {
        cudaSetDevice(dev);
        parnoldi_thread_disable(!persistent && workers > 1);
        parnoldi_thread_cta_cap(cta_cap);
        cufsp_mat *A = nullptr;
        cudaStream_t st = nullptr;
        cufsp_status s = cufsp_mat_create(desc, CUFSP_FORMAT_KRONECKER, &A);
        if (s == CUFSP_SUCCESS && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
            s = set_error(CUFSP_ERR_CUDA, "stream creation failed");
        while (s == CUFSP_SUCCESS) {
            const int i = next.fetch_add(1);
            if (i >= n_sets) break;
            s = cufsp_likelihood_grad(A, coefs + (size_t)i * nr, n_times, times, d_p0, block, d_counts, m, tol,
                                      logL + i, grad + (size_t)i * nr, (cufsp_stream_t)st);
        }
        if (s != CUFSP_SUCCESS) {
            status[w] = s;
            msg[w] = cufsp_last_error();
            next.store(n_sets);  // the other workers stop at their next set
        }
        if (st) cudaStreamDestroy(st);
        cufsp_mat_destroy(A);
        parnoldi_thread_disable(false);
        parnoldi_thread_cta_cap(0);
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < workers; ++w) pool.emplace_back(work, w);
    work(0);
    for (auto &t : pool) t.join();
    for (int w = 0; w < workers; ++w)
        if (status[w] != CUFSP_SUCCESS) return set_error(status[w], "cufsp_likelihood_grad_batched: " + msg[w]);
    return CUFSP_SUCCESS;
}
