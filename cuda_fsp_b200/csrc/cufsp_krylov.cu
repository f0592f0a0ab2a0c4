// cufsp_krylov.cu -- adaptive Krylov exp(tA)v (replaces cuFSP::KryExpvFSP,
// src/KryExpvFSP.h:20-108, src/KryExpvFSP.cu:6-203).
//
// Same algorithm as the reference (Expokit expv step control, classical Gram-Schmidt Arnoldi with
// optional incomplete orthogonalisation, augmented (m+2)x(m+2) Hessenberg matrix, phi1/phi2 error
// estimate), re-organised so that a whole Arnoldi pass runs on the device without host round trips:
//  * basis vectors are stored as W_k with v_k = rho_k W_k (rho on the device): the generator kernel
//    scales its output by rho_j read from device memory, and the normalisation pass of the reference
//    (cublasDscal, KryExpvFSP.cu:103-105) disappears;
//  * h = V^T w is one multi-vector dot kernel (each element of w read once for all j+1 dots), and
//    w -= V h is fused with the norm ||w|| (KryExpvFSP.cu:76-86 did gemv T, gemv N, nrm2);
//  * reductions finish in the last CTA (deterministic order) which also writes H(:, j), H(j+1, j),
//    rho_{j+1} and the happy-breakdown flag; kernels after a breakdown return at once;
//  * W_0 is the caller's vector itself (the reference copied it into the workspace, :60-64): the
//    final combination v = beta V F(:,0) (:165-166) reads each W_k[i] before writing v[i].
// One device->host copy of (H, rho, beta, flags) per step feeds the host step control, where the
// (m+2)^2 exponential is taken (Pade(13,13)).
// Deviations from the reference: k1 is reset every step (reference defect: KryExpvFSP.h:61), pi is
// exact (:48), a zero vector is returned unchanged, NaN/Inf and exhausted limits return errors.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "cufsp_internal.h"
#include "cufsp_reduce.cuh"

namespace cufsp {

constexpr int kMaxVec = CUFSP_MAX_KRYLOV + 1;

// Device state block (doubles, then one int flag):
//   H[(m+2)^2] | rho[m+2] | gam[m+2] | beta | avnorm | pad | pad | flag(int)
struct KState {
    double *H, *rho, *gam, *beta, *avnorm;
    double *btol;  // happy-breakdown threshold of the current pass (written by the host before the pass)
    int *flag;     // 0 ok, >0 happy breakdown at mb = flag, -1 NaN/Inf, -2 zero vector
    int mp2;
};

__global__ void __launch_bounds__(kRedThreads) k_step_begin(int64_t n, const double *__restrict__ v, KState s,
                                                            double *__restrict__ partials,
                                                            unsigned int *__restrict__ counter) {
    __shared__ RedSmem<1> sm;
    double acc[1] = {0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double t = v[i];
        acc[0] = fma(t, t, acc[0]);
    }
    if (!grid_reduce<1>(acc, 1, partials, counter, sm)) return;
    const double beta = sqrt(sm.final_[0]);
    for (int i = threadIdx.x; i < s.mp2 * s.mp2; i += blockDim.x) s.H[i] = 0.0;
    for (int i = threadIdx.x; i < s.mp2; i += blockDim.x) {
        s.rho[i] = 0.0;
        s.gam[i] = 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *s.beta = beta;
        *s.avnorm = 0.0;
        s.rho[0] = (beta > 0.0) ? 1.0 / beta : 0.0;
        *s.flag = !isfinite(beta) ? -1 : (beta == 0.0 ? -2 : 0);
    }
}

struct MVecArgs {
    const double *vec[kMaxVec];
    const double *v0;  // W_0 (the caller's vector)
    const double *W;   // W_1 .. W_{m+1}, contiguous with stride n
    double *w;
    int64_t n;
    int K;      // number of basis vectors used (istart..j)
    int kbase;  // istart
    int j;
    KState s;
    double *partials;
    unsigned int *counter;
};

// h_k = rho_k * (W_k . W_{j+1}) for k = istart..j;  H(k, j) = h_k;  gam_k = h_k * rho_k.
template <int KP>
__global__ void __launch_bounds__(kRedThreads) k_mdot(const MVecArgs a) {
    __shared__ RedSmem<KP> sm;
    if (*a.s.flag) return;
    double acc[KP];
#pragma unroll
    for (int k = 0; k < KP; ++k) acc[k] = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const double wi = a.w[i];
#pragma unroll
        for (int k = 0; k < KP; ++k)
            if (k < a.K) acc[k] = fma(__ldg(a.vec[k] + i), wi, acc[k]);
    }
    if (!grid_reduce<KP>(acc, a.K, a.partials, a.counter, sm)) return;
    for (int k = threadIdx.x; k < a.K; k += blockDim.x) {
        const int kk = a.kbase + k;
        const double r = a.s.rho[kk];
        const double h = r * sm.final_[k];
        a.s.H[kk + a.j * a.s.mp2] = h;
        a.s.gam[kk] = h * r;
    }
}

// Same result with the vectors split over groups of warps: warp w of a CTA serves the vector group
// g = w % G (vectors g*Kb .. g*Kb + Kg - 1, Kb = ceil(K / G) <= KG) over the states of slice w / G of
// the CTA's tile.  Each thread keeps KG sums instead of K, so the CTA stays at high occupancy for
// K up to 64 and every element of w is fetched from DRAM once per CTA (the G warps of a slice share
// it through L1).  With TWO, each lane takes two states 32 apart per tile, so that twice as many
// loads are in flight per thread (3 CTAs per SM instead of 4).
template <int KG, int G, bool TWO>
__global__ void __launch_bounds__(kRedThreads, TWO ? 3 : 4) k_mdot_grouped(const MVecArgs a) {
    constexpr int KP = KG * G;
    constexpr int S = kRedWarps / G;  // state slices of 32 (64 with TWO) in a CTA tile
    constexpr int L = TWO ? 64 : 32;
    static_assert(S * G == kRedWarps, "G must divide the warps of a CTA");
    __shared__ RedSmem<KP> sm;
    if (*a.s.flag) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = warp % G, slice = warp / G;
    const int Kb = (a.K + G - 1) / G;
    const int k0 = g * Kb;
    const int Kg = max(0, min(Kb, a.K - k0));
    // Basis vector kbase + k0 + kk: W_0 is the caller's vector, W_1.. are contiguous (stride n).
    const int ka = a.kbase + k0;
    const double *p_first = ka == 0 ? a.v0 : a.W + (int64_t)(ka - 1) * a.n;
    const double *p_next = a.W + (int64_t)ka * a.n;  // vector ka + 1; read only when Kg > 1
    double acc[KG];
#pragma unroll
    for (int kk = 0; kk < KG; ++kk) acc[kk] = 0.0;
    constexpr int64_t tile = (int64_t)S * L;
    const int64_t stride = (int64_t)gridDim.x * tile;
    for (int64_t i0 = (int64_t)blockIdx.x * tile + slice * L + lane; i0 < a.n; i0 += stride) {
        const int64_t i1 = i0 + 32;
        const bool two = TWO && i1 < a.n;
        const double w0 = __ldg(a.w + i0);
        const double w1 = two ? __ldg(a.w + i1) : 0.0;
        double u0[KG], u1[KG];
        if (Kg > 0) {
            u0[0] = __ldg(p_first + i0);
            u1[0] = two ? __ldg(p_first + i1) : 0.0;
        }
        const double *q = p_next + i0;
#pragma unroll
        for (int kk = 1; kk < KG; ++kk) {
            if (kk < Kg) {
                u0[kk] = __ldg(q);
                u1[kk] = two ? __ldg(q + 32) : 0.0;
                q += a.n;
            }
        }
#pragma unroll
        for (int kk = 0; kk < KG; ++kk)
            if (kk < Kg) acc[kk] = TWO ? fma(u1[kk], w1, fma(u0[kk], w0, acc[kk])) : fma(u0[kk], w0, acc[kk]);
    }
#pragma unroll
    for (int kk = 0; kk < KG; ++kk) {
        if (kk < Kg) {
            double v = acc[kk];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) sm.warp_part[warp][kk] = v;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < a.K; k += blockDim.x) {
        const int gg = k / Kb, kk = k - gg * Kb;
        double v = 0.0;
        for (int s = 0; s < S; ++s) v += sm.warp_part[s * G + gg][kk];
        a.partials[(size_t)blockIdx.x * KP + k] = v;
    }
    if (!grid_finish<KP>(a.K, a.partials, a.counter, sm)) return;
    for (int k = threadIdx.x; k < a.K; k += blockDim.x) {
        const int kk = a.kbase + k;
        const double r = a.s.rho[kk];
        const double h = r * sm.final_[k];
        a.s.H[kk + a.j * a.s.mp2] = h;
        a.s.gam[kk] = h * r;
    }
}

template <int KG, int G>
void launch_mdot_grouped(const MVecArgs &a, int mode, int sm_count, cudaStream_t st) {
    if (mode == 2) k_mdot_grouped<KG, G, true><<<3 * sm_count, kRedThreads, 0, st>>>(a);
    else k_mdot_grouped<KG, G, false><<<4 * sm_count, kRedThreads, 0, st>>>(a);
}

// W_{j+1} -= sum_k gam_k W_k;  s = rho_j-scaled norm;  H(j+1, j) = s;  rho_{j+1} = 1/s;
// happy breakdown when s < btol (src/KryExpvFSP.cu:76-105).
template <int KP>
__global__ void __launch_bounds__(kRedThreads) k_mupd(const MVecArgs a) {
    __shared__ RedSmem<1> sm;
    __shared__ double g[KP];
    if (*a.s.flag) return;
    for (int k = threadIdx.x; k < KP; k += blockDim.x) g[k] = (k < a.K) ? a.s.gam[a.kbase + k] : 0.0;
    __syncthreads();
    double acc[1] = {0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        double wi = a.w[i];
#pragma unroll
        for (int k = 0; k < KP; ++k)
            if (k < a.K) wi = fma(-g[k], __ldg(a.vec[k] + i), wi);
        a.w[i] = wi;
        acc[0] = fma(wi, wi, acc[0]);
    }
    if (!grid_reduce<1>(acc, 1, a.partials, a.counter, sm)) return;
    if (threadIdx.x == 0) {
        const double sn = sqrt(sm.final_[0]);
        if (!isfinite(sn)) {
            *a.s.flag = -1;
        } else if (sn < *a.s.btol) {
            *a.s.flag = a.j + 1;
        } else {
            a.s.H[(a.j + 1) + a.j * a.s.mp2] = sn;
            a.s.rho[a.j + 1] = 1.0 / sn;
        }
    }
}

// avnorm = ||A v_m|| (src/KryExpvFSP.cu:114-120); skipped after a breakdown.
__global__ void __launch_bounds__(kRedThreads) k_avnorm(int64_t n, const double *__restrict__ w, KState s,
                                                        double *__restrict__ partials,
                                                        unsigned int *__restrict__ counter) {
    __shared__ RedSmem<1> sm;
    if (*s.flag) return;
    double acc[1] = {0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double t = w[i];
        acc[0] = fma(t, t, acc[0]);
    }
    if (grid_reduce<1>(acc, 1, partials, counter, sm) && threadIdx.x == 0) {
        const double av = sqrt(sm.final_[0]);
        *s.avnorm = av;
        if (!isfinite(av)) *s.flag = -1;
    }
}

struct CombArgs {
    const double *vec[kMaxVec];
    double *out;  // may alias vec[0]
    int64_t n;
    int K;
    double c[kMaxVec];
};

// out = sum_k c_k W_k  (sol = beta V F(:,0), src/KryExpvFSP.cu:160-166).
template <int KP>
__global__ void __launch_bounds__(256) k_comb(const CombArgs a) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < KP; ++k)
            if (k < a.K) acc = fma(a.c[k], a.vec[k][i], acc);
        a.out[i] = acc;
    }
}

}  // namespace cufsp

using namespace cufsp;

struct cufsp_expv_s {
    int64_t n = 0;
    int m = 30;
    double tol = 1e-8;
    int iop = 0, q_iop = 2;
    double anorm = 1.0;
    int64_t max_nstep = 10000, max_reject = 1000;
    double t_final = 0.0, t_now = 0.0, t_new = 0.0, btol = 0.0, xm = 0.0;
    double *h_btol = nullptr;  // pinned host copy of the pass's breakdown threshold (copied to ks.btol)
    int64_t i_step = 0;
    cufsp_mat *A = nullptr;
    std::vector<double> coefs;
    cufsp_matvec_fn fn = nullptr;
    void *user = nullptr;
    double *W = nullptr;       // W_1 .. W_{m+1}
    double *d_state = nullptr; // KState block
    KState ks;
    size_t state_bytes = 0;
    ReduceScratch rs;
    int grid = 1;
    std::vector<double> hstate, Hh, F, tH;
    cufsp_expv_stats stats;
    bool transpose = false;      // apply A^T instead of A (adjoint solves)
    cufsp::KrylovStep last;      // basis data of the last Arnoldi pass / accepted step
    // CUDA graphs of the Arnoldi pass (generator-bound operators only), one per (vector, form)
    struct Graph {
        const double *v;
        bool avnorm, transpose;
        cudaGraphExec_t exec;
    };
    std::vector<Graph> graphs;
    cudaStream_t cap_stream = nullptr;
    cufsp::PArnoldi *pa = nullptr;  // persistent single-launch Arnoldi pass (small generators)
    // the stream of the handle's device work; released buffers wait for it alone unless several were used
    cudaStream_t last_stream = nullptr;
    bool used = false, mixed = false;
};

namespace {

inline double *wvec(cufsp_expv *E, double *v, int k) { return k == 0 ? v : E->W + (size_t)(k - 1) * E->n; }

cufsp_status matvec(cufsp_expv *E, const double *x, double *y, const double *d_alpha, cudaStream_t st) {
    if (E->A && E->transpose) return mat_apply_transpose(E->A, E->coefs.data(), 1.0, d_alpha, E->ks.flag, x, y, st);
    if (E->A) return mat_apply(E->A, E->coefs.data(), 1.0, d_alpha, E->ks.flag, x, false, y, st);
    // MVFun form (src/KryExpvFSP.h:15): the callback accumulates into a zeroed y.
    cufsp_status s = launch_fill(E->n, y, 0.0, st);
    if (s != CUFSP_SUCCESS) return s;
    if (E->fn(x, y, E->user, (cufsp_stream_t)st) != 0)
        return set_error(CUFSP_ERR_INVALID_ARG, "expv: matvec callback returned an error");
    return launch_scale(E->n, y, d_alpha, 1.0, st);
}

// Multi-vector dot kernel: CUFSP_KRYLOV_MDOT=0 one thread over all vectors (k_mdot), 1 vectors split
// over warp groups (k_mdot_grouped), 2 the same with two states per lane (default).
int mdot_mode() {
    static const int mode = [] {
        const char *e = getenv("CUFSP_KRYLOV_MDOT");
        const int v = e ? atoi(e) : 2;
        return v < 0 || v > 2 ? 2 : v;
    }();
    return mode;
}

template <int KP>
void launch_mdot(const MVecArgs &a, int grid, cudaStream_t st) { k_mdot<KP><<<grid, kRedThreads, 0, st>>>(a); }
template <int KP>
void launch_mupd(const MVecArgs &a, int grid, cudaStream_t st) { k_mupd<KP><<<grid, kRedThreads, 0, st>>>(a); }
template <int KP>
void launch_comb(const CombArgs &a, int grid, cudaStream_t st) { k_comb<KP><<<grid, 256, 0, st>>>(a); }

cufsp_status arnoldi_dot_update(cufsp_expv *E, double *v, int j, int istart, cudaStream_t st) {
    MVecArgs a;
    a.K = j - istart + 1;
    a.kbase = istart;
    for (int k = 0; k < a.K; ++k) a.vec[k] = wvec(E, v, istart + k);
    a.v0 = v;
    a.W = E->W;
    a.w = wvec(E, v, j + 1);
    a.n = E->n;
    a.j = j;
    a.s = E->ks;
    a.partials = E->rs.partials;
    a.counter = E->rs.counter;
    const int K = a.K;
    const int mode = mdot_mode();
    const int sms = device_info().sm_count;
    if (mode == 0 || E->grid < 4 * sms) {  // small vectors: the grid of the other pass kernels
        if (K <= 8) launch_mdot<8>(a, E->grid, st);
        else if (K <= 16) launch_mdot<16>(a, E->grid, st);
        else if (K <= 32) launch_mdot<32>(a, E->grid, st);
        else launch_mdot<64>(a, E->grid, st);
    } else if (K <= 8) {
        launch_mdot_grouped<8, 1>(a, mode, sms, st);
    } else if (K <= 16) {
        launch_mdot_grouped<8, 2>(a, mode, sms, st);
    } else if (K <= 32) {
        launch_mdot_grouped<8, 4>(a, mode, sms, st);
    } else {
        launch_mdot_grouped<8, 8>(a, mode, sms, st);
    }
    CUFSP_CUDA_TRY(cudaGetLastError());
    if (K <= 8) launch_mupd<8>(a, E->grid, st);
    else if (K <= 16) launch_mupd<16>(a, E->grid, st);
    else if (K <= 32) launch_mupd<32>(a, E->grid, st);
    else launch_mupd<64>(a, E->grid, st);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

// The Arnoldi pass of one step, entirely on the device (src/KryExpvFSP.cu:38-120): basis
// W_1..W_{m+1} (W_0 = v), Hessenberg matrix, rho, beta, ||A v_m|| (when with_avnorm), breakdown
// flag; one device->host copy of the state block into E->hstate.
// The launches of one Arnoldi pass on stream st (no synchronisation).
cufsp_status arnoldi_launches(cufsp_expv *E, double *v, cudaStream_t st, bool with_avnorm) {
    const int m = E->m;
    k_step_begin<<<E->grid, kRedThreads, 0, st>>>(E->n, v, E->ks, E->rs.partials, E->rs.counter);
    CUFSP_CUDA_TRY(cudaGetLastError());
    cufsp_status s;
    int istart = 0;
    for (int j = 0; j < m; ++j) {
        s = matvec(E, wvec(E, v, j), wvec(E, v, j + 1), E->ks.rho + j, st);
        if (s != CUFSP_SUCCESS) return s;
        if (E->iop) istart = (j >= E->q_iop - 1) ? j - E->q_iop + 1 : 0;
        s = arnoldi_dot_update(E, v, j, istart, st);
        if (s != CUFSP_SUCCESS) return s;
    }
    if (with_avnorm) {
        s = matvec(E, wvec(E, v, m), wvec(E, v, m + 1), E->ks.rho + m, st);
        if (s != CUFSP_SUCCESS) return s;
        k_avnorm<<<E->grid, kRedThreads, 0, st>>>(E->n, wvec(E, v, m + 1), E->ks, E->rs.partials, E->rs.counter);
        CUFSP_CUDA_TRY(cudaGetLastError());
    }
    return CUFSP_SUCCESS;
}

// The state block travels to the host once per pass: a one-CTA kernel copies it into pinned host
// memory (reachable from the device through unified addressing) and raises a sequence word that the
// host polls, instead of a copy command and a stream synchronisation.  The poll is bounded: the
// stream is queried every 1024 polls, and a finished or failed stream, or 10 s, ends it; a
// synchronisation then returns any error.  The pinned buffer is per host thread (calls are
// synchronous, so one buffer serves every driver of the thread).  CUFSP_KRYLOV_SPIN=0: a copy and a
// synchronisation.
__global__ void k_publish_state(const double *__restrict__ d, double *h, int words, unsigned *h_seq, unsigned seq) {
    for (int k = threadIdx.x; k < words; k += blockDim.x) h[k] = d[k];
    __threadfence_system();
    __syncthreads();
    if (threadIdx.x == 0) *(volatile unsigned *)h_seq = seq;
}

struct PinnedState {
    double *p = nullptr;
    unsigned *seq = nullptr;
    size_t bytes = 0;
    unsigned n = 0;
    ~PinnedState() {
        if (p) cudaFreeHost(p);
        if (seq) cudaFreeHost(seq);
    }
};
thread_local PinnedState tl_pin;

bool spin_state() {
    static const bool on = [] {
        const char *e = getenv("CUFSP_KRYLOV_SPIN");
        return !e || atoi(e) != 0;
    }();
    return on;
}

cufsp_status fetch_state(cufsp_expv *E, cudaStream_t st) {
    bool spin = spin_state();
    if (spin && tl_pin.bytes < E->state_bytes) {
        if (tl_pin.p) cudaFreeHost(tl_pin.p);
        tl_pin.p = nullptr;
        tl_pin.bytes = 0;
        if (!tl_pin.seq && cudaHostAlloc((void **)&tl_pin.seq, 64, cudaHostAllocPortable | cudaHostAllocMapped) != cudaSuccess)
            tl_pin.seq = nullptr;
        if (tl_pin.seq &&
            cudaHostAlloc((void **)&tl_pin.p, E->state_bytes, cudaHostAllocPortable | cudaHostAllocMapped) == cudaSuccess) {
            tl_pin.bytes = E->state_bytes;
            *(volatile unsigned *)tl_pin.seq = tl_pin.n;
        } else {
            cudaGetLastError();
            tl_pin.p = nullptr;
            spin = false;
        }
    }
    if (!spin) {
        CUFSP_CUDA_TRY(cudaMemcpyAsync(E->hstate.data(), E->d_state, E->state_bytes, cudaMemcpyDeviceToHost, st));
        CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
        return CUFSP_SUCCESS;
    }
    const unsigned seq = ++tl_pin.n;
    const int words = (int)(E->state_bytes / sizeof(double));
    k_publish_state<<<1, 256, 0, st>>>(E->d_state, tl_pin.p, words, tl_pin.seq, seq);
    CUFSP_CUDA_TRY(cudaGetLastError());
    const auto t0 = std::chrono::steady_clock::now();
    for (unsigned it = 1; *(volatile unsigned *)tl_pin.seq != seq; ++it) {
        if ((it & 1023) == 0) {
            if (cudaStreamQuery(st) != cudaErrorNotReady) break;
            if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(10)) break;
        }
    }
    if (*(volatile unsigned *)tl_pin.seq != seq) CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
    std::memcpy(E->hstate.data(), tl_pin.p, E->state_bytes);
    return CUFSP_SUCCESS;
}

bool graphs_enabled() {
    static const bool on = [] {
        const char *e = getenv("CUFSP_KRYLOV_GRAPH");
        return !e || atoi(e) != 0;
    }();
    return on;
}

// The Arnoldi pass of one step, entirely on the device (src/KryExpvFSP.cu:38-120): basis
// W_1..W_{m+1} (W_0 = v), Hessenberg matrix, rho, beta, ||A v_m|| (when with_avnorm), breakdown
// flag; one device->host copy of the state block into E->hstate.  With a generator bound, the ~3m
// launches are captured once per (vector, form) into a CUDA graph and replayed (one launch per
// step); the generator's coefficient-dependent tables are prepared eagerly before each replay.
// btol_eff: happy-breakdown threshold of this pass.
cufsp_status arnoldi_pass(cufsp_expv *E, double *v, cudaStream_t st, bool with_avnorm, double btol_eff) {
    cufsp_status s;
    if (E->used && E->last_stream != st) E->mixed = true;
    E->used = true;
    E->last_stream = st;
    const bool persistent = E->A && parnoldi_wanted(E->A, E->n, E->m);
    if (persistent) {
        s = parnoldi_run(&E->pa, E->A, E->coefs, E->transpose, E->n, v, E->W, E->ks.H, E->ks.rho, E->ks.gam,
                         E->ks.beta, E->ks.avnorm, E->ks.flag, E->ks.flag + 1, E->m, E->iop, E->q_iop, btol_eff,
                         with_avnorm, st);
        if (s != CUFSP_SUCCESS) return s;
    } else if (E->A && graphs_enabled()) {
        *E->h_btol = btol_eff;  // the previous pass's copy has completed: the stream was synchronised after it
        CUFSP_CUDA_TRY(cudaMemcpyAsync(E->ks.btol, E->h_btol, sizeof(double), cudaMemcpyHostToDevice, st));
        s = mat_prepare(E->A, E->coefs.data(), st, E->transpose);
        if (s != CUFSP_SUCCESS) return s;
        cudaGraphExec_t exec = nullptr;
        for (auto &g : E->graphs)
            if (g.v == v && g.avnorm == with_avnorm && g.transpose == E->transpose) exec = g.exec;
        if (!exec) {
            if (!E->cap_stream) CUFSP_CUDA_TRY(cudaStreamCreateWithFlags(&E->cap_stream, cudaStreamNonBlocking));
            cudaGraph_t graph = nullptr;
            CUFSP_CUDA_TRY(cudaStreamBeginCapture(E->cap_stream, cudaStreamCaptureModeThreadLocal));
            s = arnoldi_launches(E, v, E->cap_stream, with_avnorm);
            const cudaError_t e = cudaStreamEndCapture(E->cap_stream, &graph);
            if (s != CUFSP_SUCCESS) {
                if (graph) cudaGraphDestroy(graph);
                return s;
            }
            if (e != cudaSuccess) return cuda_error(e, "expv: graph capture");
            const cudaError_t e2 = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (e2 != cudaSuccess) return cuda_error(e2, "expv: graph instantiate");
            if (E->graphs.size() >= 4) {  // a small cache; the oldest entry goes
                cudaGraphExecDestroy(E->graphs.front().exec);
                E->graphs.erase(E->graphs.begin());
            }
            E->graphs.push_back({v, with_avnorm, E->transpose, exec});
        }
        CUFSP_CUDA_TRY(cudaGraphLaunch(exec, st));
    } else {
        *E->h_btol = btol_eff;
        CUFSP_CUDA_TRY(cudaMemcpyAsync(E->ks.btol, E->h_btol, sizeof(double), cudaMemcpyHostToDevice, st));
        s = arnoldi_launches(E, v, st, with_avnorm);
        if (s != CUFSP_SUCCESS) return s;
    }
    const int m = E->m;
    s = fetch_state(E, st);
    if (s != CUFSP_SUCCESS) return s;
    // basis data for the adjoint (leading mb x mb block of H, rho, beta)
    const int mp2 = m + 2;
    const double *hH = E->hstate.data();
    const double *hrho = hH + (size_t)mp2 * mp2;
    int flag, barrier_err;
    std::memcpy(&flag, hrho + 2 * mp2 + 4, sizeof(int));
    std::memcpy(&barrier_err, reinterpret_cast<const char *>(hrho + 2 * mp2 + 4) + sizeof(int), sizeof(int));
    if (persistent && barrier_err)
        return set_error(CUFSP_ERR_CUDA, "expv: a grid barrier wait of the persistent Arnoldi pass expired");
    if (!persistent && E->A) {
        s = mat_check_watchdog(E->A, "expv");
        if (s != CUFSP_SUCCESS) return s;
    }
    KrylovStep &L = E->last;
    L.mb = flag > 0 ? flag : m;
    L.beta = hrho[2 * mp2];
    L.H.assign((size_t)L.mb * L.mb, 0.0);
    for (int j = 0; j < L.mb; ++j)
        for (int i = 0; i < L.mb; ++i) L.H[i + (size_t)j * L.mb] = hH[i + (size_t)j * mp2];
    L.rho.assign(hrho, hrho + L.mb);
    L.tau = 0.0;
    return CUFSP_SUCCESS;
}

double round2(double t) {
    const double s = std::pow(10.0, std::floor(std::log10(t)) - 1.0);
    return std::ceil(t / s) * s;
}

cufsp_status expv_step(cufsp_expv *E, double *v, cudaStream_t st) {
    if (!E->A && !E->fn) return set_error(CUFSP_ERR_INVALID_ARG, "expv: no operator bound");
    if (E->t_now >= E->t_final) return CUFSP_SUCCESS;
    if (E->i_step >= E->max_nstep) return set_error(CUFSP_ERR_STEP_LIMIT, "expv: max_nstep reached");
    const int m = E->m, mp2 = m + 2;
    const double delta = 1.2, gamma = 0.9;
    if (E->i_step == 0) E->btol = E->anorm * E->tol;  // tolerance for happy breakdown (:50)

    // A happy breakdown ends the solve in one jump to t_final (:90-98) whose error grows like the
    // residual times the remaining time; the reference accepts residuals below anorm * tol, i.e. an
    // error of up to tol per unit of the remaining time.  Dividing the threshold by the remaining
    // time (when above 1) keeps the jump's error within tol.
    const double btol_eff = E->btol / std::max(1.0, E->t_final - E->t_now);
    cufsp_status s = arnoldi_pass(E, v, st, true, btol_eff);
    if (s != CUFSP_SUCCESS) return s;
    const double *hH = E->hstate.data();
    const double *hrho = hH + (size_t)mp2 * mp2;
    const double beta = hrho[2 * mp2];
    const double avnorm = hrho[2 * mp2 + 1];
    int flag;
    std::memcpy(&flag, hrho + 2 * mp2 + 4, sizeof(int));
    if (flag == -2) {  // zero vector: exp(tA) 0 = 0
        E->t_now = E->t_final;
        E->last.tau = 0.0;
        E->last.beta = 0.0;
        return CUFSP_SUCCESS;
    }
    if (flag == -1) return set_error(CUFSP_ERR_NONFINITE, "expv: NaN/Inf in the Krylov iteration");

    if (E->i_step == 0) {  // first-step size, src/KryExpvFSP.cu:45-51
        E->xm = 1.0 / (double)m;
        const double fact = std::pow((m + 1) / std::exp(1.0), m + 1) * std::sqrt(2.0 * M_PI * (m + 1));
        E->t_new = (1.0 / E->anorm) * std::pow((fact * E->tol) / (4.0 * beta * E->anorm), E->xm);
    }
    int mb = m, k1 = 2;
    double tau = std::min(E->t_final - E->t_now, E->t_new);
    int64_t n_mv = m + 1;
    if (flag > 0) {  // happy breakdown (:90-98)
        k1 = 0;
        mb = flag;
        tau = E->t_final - E->t_now;
        n_mv = mb;
        E->stats.n_breakdown++;
    }
    E->stats.n_matvec += n_mv;
    std::memcpy(E->Hh.data(), hH, sizeof(double) * mp2 * mp2);
    if (k1 != 0) E->Hh[(m + 1) + (size_t)m * mp2] = 1.0;

    double err_loc = 0.0;
    int64_t ireject = 0;
    bool accepted = false;
    while (ireject < E->max_reject) {  // rejection loop, :122-158
        const int mx = mb + k1;
        for (int i = 0; i < mp2 * mp2; ++i) E->tH[i] = tau * E->Hh[i];
        s = expm_pade13(mp2, E->tH.data(), E->F.data());
        if (s != CUFSP_SUCCESS) return s;
        if (k1 == 0) {
            err_loc = E->btol;
            accepted = true;
            break;
        }
        const double phi1 = std::fabs(beta * E->F[mx - 2]);
        const double phi2 = std::fabs(beta * E->F[mx - 1] * avnorm);
        if (phi1 > phi2 * 10.0) {
            err_loc = phi2;
            E->xm = 1.0 / (double)mx;
        } else if (phi1 > phi2) {
            err_loc = (phi1 * phi2) / (phi1 - phi2);
            E->xm = 1.0 / (double)mx;
        } else {
            err_loc = phi1;
            E->xm = 1.0 / (double)(mx - 1);
        }
        if (!std::isfinite(err_loc)) return set_error(CUFSP_ERR_NONFINITE, "expv: non-finite error estimate");
        if (err_loc <= delta * tau * E->tol) {
            accepted = true;
            break;
        }
        tau = round2(gamma * tau * std::pow(tau * E->tol / err_loc, E->xm));
        ++ireject;
        E->stats.n_reject++;
    }
    if (!accepted) return set_error(CUFSP_ERR_STEP_LIMIT, "expv: max_reject reached");

    // v = beta * V[:, 0:mx] F(0:mx, 0) = sum_k (beta F_k0 rho_k) W_k
    const int mx = mb + std::max(0, k1 - 1);
    CombArgs c;
    c.K = mx;
    c.n = E->n;
    c.out = v;
    for (int k = 0; k < mx; ++k) {
        c.vec[k] = wvec(E, v, k);
        c.c[k] = beta * E->F[k] * hrho[k];
    }
    const int g = stream_grid(E->n, 4, device_info().sm_count * 8);
    if (mx <= 8) launch_comb<8>(c, g, st);
    else if (mx <= 16) launch_comb<16>(c, g, st);
    else if (mx <= 32) launch_comb<32>(c, g, st);
    else launch_comb<64>(c, g, st);
    CUFSP_CUDA_TRY(cudaGetLastError());

    const bool last = (tau >= E->t_final - E->t_now);
    E->last.tau = last ? E->t_final - E->t_now : tau;
    E->t_now = last ? E->t_final : E->t_now + tau;
    if (err_loc > 0.0) E->t_new = round2(gamma * tau * std::pow(tau * E->tol / err_loc, E->xm));
    if (!(E->t_new > 0.0) || !std::isfinite(E->t_new)) E->t_new = E->t_final - E->t_now;
    E->i_step++;
    E->stats.n_steps++;
    E->stats.t_now = E->t_now;
    E->stats.last_err = err_loc;
    return CUFSP_SUCCESS;
}

}  // namespace

namespace cufsp {
void expv_set_transpose(cufsp_expv *E, bool transpose) { E->transpose = transpose; }
cufsp_status expv_arnoldi(cufsp_expv *E, double *v, cudaStream_t st) {
    return arnoldi_pass(E, v, st, false, E->btol > 0.0 ? E->btol : E->anorm * E->tol);
}
cufsp_status expv_step_once(cufsp_expv *E, double *v, cudaStream_t st) { return expv_step(E, v, st); }
const KrylovStep &expv_last(const cufsp_expv *E) { return E->last; }
const double *expv_basis(const cufsp_expv *E, const double *v, int k) {
    return k == 0 ? v : E->W + (size_t)(k - 1) * E->n;
}
}  // namespace cufsp

extern "C" cufsp_status cufsp_expv_create(int64_t n, int m, double tol, int iop, int q_iop, double anorm,
                                          cufsp_expv **out) {
    clear_error();
    if (!out) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_create: out is NULL");
    *out = nullptr;
    if (n < 1 || n > 2147483647LL) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_create: n out of range");
    if (m < 1 || m > CUFSP_MAX_KRYLOV) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_create: m must be in [1, 60]");
    if (!(tol > 0.0) || !(anorm > 0.0)) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_create: tol and anorm must be > 0");
    if (iop && q_iop < 1) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_create: q_iop must be >= 1");
    cufsp_expv *E = new cufsp_expv();
    E->n = n;
    E->m = m;
    E->tol = tol;
    E->iop = iop;
    E->q_iop = q_iop;
    E->anorm = anorm;
    const int mp2 = m + 2;
    const size_t nd = (size_t)mp2 * mp2 + 2 * (size_t)mp2 + 4;
    E->state_bytes = nd * sizeof(double) + 2 * sizeof(int);
    E->hstate.resize(nd + 1);
    E->Hh.resize((size_t)mp2 * mp2);
    E->F.resize((size_t)mp2 * mp2);
    E->tH.resize((size_t)mp2 * mp2);
    std::memset(&E->stats, 0, sizeof(E->stats));
    cudaError_t e = cache_alloc((void **)&E->W, sizeof(double) * (size_t)n * (size_t)(m + 1));
    if (e == cudaSuccess) e = cache_alloc((void **)&E->d_state, E->state_bytes);
    if (e == cudaSuccess) e = cudaMemset(E->d_state, 0, E->state_bytes);
    if (e == cudaSuccess) e = upload_fence();
    if (e != cudaSuccess) {
        cufsp_expv_destroy(E);
        return cuda_error(e, "cufsp_expv_create");
    }
    double *b = E->d_state;
    E->ks.H = b;
    E->ks.rho = b + (size_t)mp2 * mp2;
    E->ks.gam = E->ks.rho + mp2;
    E->ks.beta = E->ks.gam + mp2;
    E->ks.avnorm = E->ks.beta + 1;
    E->ks.btol = E->ks.beta + 2;
    E->ks.flag = reinterpret_cast<int *>(E->ks.beta + 4);
    if (!(E->h_btol = pinned_slot_get())) {
        cufsp_expv_destroy(E);
        return set_error(CUFSP_ERR_ALLOC, "cufsp_expv_create: pinned allocation failed");
    }
    E->ks.mp2 = mp2;
    E->grid = stream_grid(n, 4, device_info().sm_count * 4);
    cufsp_status s = E->rs.init(E->grid, 64);
    if (s != CUFSP_SUCCESS) {
        cufsp_expv_destroy(E);
        return s;
    }
    *out = E;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_expv_destroy(cufsp_expv *E) {
    if (!E) return CUFSP_SUCCESS;
    for (auto &g : E->graphs) cudaGraphExecDestroy(g.exec);
    if (E->used && !E->mixed) {  // every launch of the handle was ordered on one stream
        parnoldi_destroy(E->pa, E->last_stream);
        cache_free(E->W, E->last_stream);
        cache_free(E->d_state, E->last_stream);
        E->rs.release(E->last_stream);
    } else {
        parnoldi_destroy(E->pa);
        cache_free(E->W);
        cache_free(E->d_state);
        E->rs.release();
    }
    if (E->cap_stream) cudaStreamDestroy(E->cap_stream);
    // every copy from h_btol completed inside the call that issued it (each pass ends with a blocking
    // read of its state block), so the slot is free for the next driver
    pinned_slot_put(E->h_btol);
    delete E;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_expv_set_limits(cufsp_expv *E, int64_t max_nstep, int64_t max_reject) {
    if (!E || max_nstep < 1 || max_reject < 1) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_set_limits: bad argument");
    E->max_nstep = max_nstep;
    E->max_reject = max_reject;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_expv_bind_mat_coefs(cufsp_expv *E, cufsp_mat *A, const double *coefs) {
    if (!E || !A) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_bind_mat: NULL argument");
    int64_t n = 0;
    cufsp_mat_num_states(A, &n);
    if (n != E->n) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_bind_mat: size mismatch");
    cufsp_status s = mat_coefs(A, 0.0, coefs, E->coefs);
    if (s != CUFSP_SUCCESS) return s;
    // graphs hold the operator's launch parameters (coefficients included): rebuild them
    for (auto &g : E->graphs) cudaGraphExecDestroy(g.exec);
    E->graphs.clear();
    if (E->A != A) {  // the persistent pass keeps the generator's model data
        parnoldi_destroy(E->pa);
        E->pa = nullptr;
    }
    E->A = A;
    E->fn = nullptr;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_expv_bind_mat(cufsp_expv *E, cufsp_mat *A, double t_mat) {
    if (!E || !A) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_bind_mat: NULL argument");
    std::vector<double> c;
    cufsp_status s = mat_coefs(A, t_mat, nullptr, c);
    if (s != CUFSP_SUCCESS) return s;
    return cufsp_expv_bind_mat_coefs(E, A, c.data());
}

extern "C" cufsp_status cufsp_expv_bind_matvec(cufsp_expv *E, cufsp_matvec_fn fn, void *user) {
    if (!E || !fn) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_bind_matvec: NULL argument");
    E->fn = fn;
    E->user = user;
    E->A = nullptr;
    for (auto &g : E->graphs) cudaGraphExecDestroy(g.exec);
    E->graphs.clear();
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_expv_set_final_time(cufsp_expv *E, double t_final) {
    if (!E || !(t_final >= 0.0) || !std::isfinite(t_final))
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_set_final_time: bad argument");
    E->t_final = t_final;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_expv_step(cufsp_expv *E, double *v, cufsp_stream_t stream) {
    if (!E || !v) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_step: NULL argument");
    return expv_step(E, v, (cudaStream_t)stream);
}

extern "C" cufsp_status cufsp_expv_solve(cufsp_expv *E, double *v, cufsp_stream_t stream, cufsp_expv_stats *stats) {
    if (!E || !v) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_solve: NULL argument");
    cufsp_status s = CUFSP_SUCCESS;
    while (E->t_now < E->t_final) {  // KryExpvFSP::solve, src/KryExpvFSP.cu:184-188
        s = expv_step(E, v, (cudaStream_t)stream);
        if (s != CUFSP_SUCCESS) break;
    }
    if (s == CUFSP_SUCCESS) {
        cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
        if (e != cudaSuccess) s = cuda_error(e, "cufsp_expv_solve");
    }
    if (stats) *stats = E->stats;
    return s;
}

extern "C" cufsp_status cufsp_expv_reset_time(cufsp_expv *E) {
    if (!E) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_reset_time: NULL argument");
    E->t_now = 0.0;  // the current vector is kept (src/KryExpvFSP.h:82-84)
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_expv_final_time_reached(const cufsp_expv *E, int *reached) {
    if (!E || !reached) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_final_time_reached: NULL argument");
    *reached = E->t_now >= E->t_final;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_expv_get_stats(const cufsp_expv *E, cufsp_expv_stats *stats) {
    if (!E || !stats) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_expv_get_stats: NULL argument");
    *stats = E->stats;
    return CUFSP_SUCCESS;
}
