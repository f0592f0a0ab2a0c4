// cufsp_batch.cuh -- batched adaptive Krylov exp(tA)p over many FSP instances in ONE persistent launch.
//
// The single-instance Krylov driver (cufsp_krylov.cu, replacing cuFSP::KryExpvFSP,
// src/KryExpvFSP.cu:38-188) runs its step control on the host, one synchronisation per step.  Here
// every part of the solve runs on the device, for hundreds of instances of one reaction network that
// differ in their box (truncation bounds), their factor tables and their rate coefficients:
//  * Work split: the grid is a set of thread-block clusters; each cluster takes instances from a
//    global work counter (largest first) and solves one instance at a time with all its CTAs.  The
//    cluster's CTAs split the instance's states into contiguous chunks.
//  * Reductions (norms, the Gram-Schmidt dots) go through distributed shared memory: every CTA
//    writes its partial sums, one cluster barrier (barrier.cluster: hardware, no spinning), then
//    every CTA sums the partials of all CTAs in rank order -- identical, deterministic results in all
//    CTAs, so every CTA holds the same Hessenberg matrix and takes the same step-control decisions
//    without further communication.
//  * Per Arnoldi iteration: the generator action w = rho_j A W_j fused with the dots of w against the
//    basis (one pass over the own chunk), a cluster reduction, the update w -= V h fused with ||w||^2,
//    a second cluster reduction.  The basis is stored unnormalised (v_k = rho_k W_k) as in the
//    single-instance driver.
//  * The small (m+2)^2 exponential is Pade(13,13) with scaling and squaring (Higham 2005, the same
//    algorithm as the host path cufsp_expm.cpp), computed by every CTA in its shared memory; the
//    Expokit step control (delta = 1.2, gamma = 0.9, phi1/phi2 estimate, 2-significant-digit
//    rounding, first-step formula) follows the host driver.
//  * Every loop is bounded (max steps and rejections per instance); an instance that exhausts them
//    or meets NaN/Inf gets an error status and the cluster moves on.  There are no spin waits.
//
// This file is compiled by NVRTC per reaction network (cufsp_batch.cu writes the prefix): species and
// reaction counts, the Krylov dimension M, the threads per CTA, and per reaction and species the net
// change nu(r, s) and the factor kind(r, s) (0: f = 1, 1: f(x) = x, 2: table lookup) are constants.

#ifndef CUFSP_BATCH_CUH
#define CUFSP_BATCH_CUH

#define CUFSP_BATCH_MAXS 8
#define CUFSP_BATCH_MAXR 32

struct CufspBatchDiv {  // unsigned division by a runtime constant d (round-up multiplier method)
    unsigned d, mul, shift;
};

struct CufspBatchInst {
    long long off;       // offset of the instance's vector in the packed array
    long long tab;       // offset of its factor tables in the packed table array
    int n;               // states
    int tab_stride;      // sum_s (b_s + 1)
    int dims[CUFSP_BATCH_MAXS];
    int tab_off[CUFSP_BATCH_MAXS];
    int delta[CUFSP_BATCH_MAXR];  // flat shift of reaction r: sum_s nu_{r,s} stride_s
    CufspBatchDiv div[CUFSP_BATCH_MAXS];
    double coef[CUFSP_BATCH_MAXR];
};

struct CufspBatchStat {
    double t;            // time reached
    double err;          // last local error estimate
    int steps, rejects, matvecs, status;  // status: 0 ok, 1 step limit, 2 NaN/Inf
};

struct CufspBatchArgs {
    const CufspBatchInst *inst;
    const int *order;        // processing order (largest instances first)
    const double *tables;    // packed factor tables
    double *p;               // packed state vectors (in: p(0), out: p(t_final))
    double *work;            // per-cluster basis workspace, work_stride doubles each
    long long work_stride;   // >= (M + 1) * max n
    unsigned *counter;       // work counter (zero before the launch)
    CufspBatchStat *stats;   // per instance
    int n_inst;
    int max_steps, max_reject;
    double t_final, tol, anorm;
};

#ifdef __CUDACC_RTC__

#include <cooperative_groups.h>
namespace cg = cooperative_groups;

namespace cufsp_batch {

constexpr int NS = CUFSP_BATCH_NS;
constexpr int NR = CUFSP_BATCH_NR;
constexpr int M = CUFSP_BATCH_M;          // Krylov dimension
constexpr int MP2 = M + 2;
constexpr int T = CUFSP_BATCH_THREADS;    // threads per CTA
constexpr int WARPS = T / 32;
constexpr int KR = M + 1;                 // most partial sums one reduction carries
constexpr bool IOP = CUFSP_BATCH_IOP != 0;
constexpr int QIOP = CUFSP_BATCH_QIOP;

// Generated: nu(r, s) and kind(r, s), constexpr functions of constant indices.

__device__ __forceinline__ unsigned fdiv(unsigned n, const CufspBatchDiv &f) {
    const unsigned t = __umulhi(n, f.mul);
    return (t + n) >> f.shift;
}

// ---- per-CTA shared state -------------------------------------------------------------------
struct Shared {
    double red[2][KR];          // this CTA's partial sums (double-buffered; read remotely)
    double warp_part[WARPS][KR];
    double tot[KR];             // cluster totals
    double H[MP2 * MP2];        // Hessenberg matrix (column-major), identical in every CTA
    double rho[MP2], gam[MP2];
    double pade[8][MP2 * MP2];  // exponential workspace
    double coefc[MP2];          // combination coefficients
    int piv[MP2];
    CufspBatchInst in;          // current instance
    int inst_idx;
    double sc[8];               // scalars broadcast inside the CTA
    int flag[4];
};

// Cluster-wide sum of one value per thread: every CTA ends with the total in s.tot[0].
__device__ __forceinline__ void cluster_sum1(cg::cluster_group &cl, Shared &s, double v, int &buf);

// Constants of the current instance, copied into registers for the generator action.
struct Regs {
    double coef[NR];
    int delta[NR];
    int dims[NS];
    CufspBatchDiv div[NS];
    int tab_off[NS];
    int tab_stride;
};

__device__ __forceinline__ void load_regs(const CufspBatchInst &in, Regs &g) {
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        g.coef[r] = in.coef[r];
        g.delta[r] = in.delta[r];
    }
#pragma unroll
    for (int sp = 0; sp < NS; ++sp) {
        g.dims[sp] = in.dims[sp];
        g.div[sp] = in.div[sp];
        g.tab_off[sp] = in.tab_off[sp];
    }
    g.tab_stride = in.tab_stride;
}

// Factor f_{r,s}(x) of the current instance.
template <int R, int SP>
__device__ __forceinline__ double factor(const Regs &g, const double *__restrict__ tab, int x) {
    if constexpr (kind(R, SP) == 0) return 1.0;
    else if constexpr (kind(R, SP) == 1) return (double)x;
    else return __ldg(tab + R * g.tab_stride + g.tab_off[SP] + x);
}

template <int R, int SP>
__device__ __forceinline__ void src_factor(const Regs &g, const double *__restrict__ tab, const int (&x)[NS], double &f,
                                           bool &ok) {
    if constexpr (SP < NS) {
        const int xs = x[SP] - nu(R, SP);
        if constexpr (nu(R, SP) > 0) ok = ok && xs >= 0;
        if constexpr (nu(R, SP) < 0) ok = ok && xs < g.dims[SP];
        if constexpr (kind(R, SP) != 0) f *= factor<R, SP>(g, tab, min(max(xs, 0), g.dims[SP] - 1));
        src_factor<R, SP + 1>(g, tab, x, f, ok);
    }
}

template <int R, int SP>
__device__ __forceinline__ void own_factor(const Regs &g, const double *__restrict__ tab, const int (&x)[NS], double &f) {
    if constexpr (SP < NS) {
        if constexpr (kind(R, SP) != 0) f *= factor<R, SP>(g, tab, x[SP]);
        own_factor<R, SP + 1>(g, tab, x, f);
    }
}

// (A v)[i] for one state: sum_r c_r (a_r(x - nu_r) v[i - d_r] 1{x - nu_r in box} - a_r(x) v[i]).
template <int R>
__device__ __forceinline__ void accumulate(const Regs &g, const double *__restrict__ tab, const double *__restrict__ v,
                                           int i, const int (&x)[NS], double vi, double &acc, double &dg) {
    if constexpr (R < NR) {
        double fa = g.coef[R], fb = g.coef[R];
        bool ok = true;
        src_factor<R, 0>(g, tab, x, fa, ok);
        own_factor<R, 0>(g, tab, x, fb);
        const double src = ok ? __ldg(v + i - g.delta[R]) : 0.0;
        acc = fma(ok ? fa : 0.0, src, acc);
        dg += fb;
        accumulate<R + 1>(g, tab, v, i, x, vi, acc, dg);
    }
}

__device__ __forceinline__ void decode(const Regs &g, int i, int (&x)[NS]) {
    unsigned rem = (unsigned)i;
#pragma unroll
    for (int sp = 0; sp < NS - 1; ++sp) {
        const unsigned q = fdiv(rem, g.div[sp]);
        x[sp] = (int)(rem - q * (unsigned)g.dims[sp]);
        rem = q;
    }
    x[NS - 1] = (int)rem;
}

// rho * (A v)[i]
__device__ __forceinline__ double apply_at(const Regs &g, const double *__restrict__ tab, const double *__restrict__ v,
                                           int i, double rho) {
    int x[NS];
    decode(g, i, x);
    const double vi = __ldg(v + i);
    double acc = 0.0, dg = 0.0;
    accumulate<0>(g, tab, v, i, x, vi, acc, dg);
    return rho * fma(-dg, vi, acc);
}

// Warp partial sums of up to 8 values into s.warp_part[warp][k0 + k].
__device__ __forceinline__ void warp_partials8(Shared &s, const double (&acc)[8], int k0, int kused) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        if (k0 + k < kused) {
            double v = acc[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) s.warp_part[warp][k0 + k] = v;
        }
    }
}

// CTA totals of s.warp_part[.][0..kused) into s.red[buf], one cluster barrier, then every CTA sums
// the partials of all CTAs in rank order into s.tot.
__device__ __forceinline__ void cluster_finish(cg::cluster_group &cl, Shared &s, int kused, int &buf) {
    __syncthreads();
    for (int k = threadIdx.x; k < kused; k += T) {
        double v = 0.0;
        for (int w = 0; w < WARPS; ++w) v += s.warp_part[w][k];
        s.red[buf][k] = v;
    }
    cl.sync();
    const int nb = (int)cl.num_blocks();
    for (int k = threadIdx.x; k < kused; k += T) {
        double v = 0.0;
        for (int b = 0; b < nb; ++b) v += cl.map_shared_rank(&s.red[buf][0], b)[k];
        s.tot[k] = v;
    }
    __syncthreads();
    buf ^= 1;
}

__device__ __forceinline__ void cluster_sum1(cg::cluster_group &cl, Shared &s, double v, int &buf) {
    double acc[8] = {v, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    warp_partials8(s, acc, 0, 1);
    cluster_finish(cl, s, 1, buf);
}

// ---- small dense kernels for the (m+2)^2 exponential (column-major, k = MP2) -------------------
__device__ void mm(const double *A, const double *B, double *C) {  // C = A B
    for (int e = threadIdx.x; e < MP2 * MP2; e += T) {
        const int i = e % MP2, j = e / MP2;
        double acc = 0.0;
        for (int l = 0; l < MP2; ++l) acc = fma(A[i + l * MP2], B[l + j * MP2], acc);
        C[e] = acc;
    }
    __syncthreads();
}

// F = exp(A) by scaling and squaring Pade(13,13); false on NaN/Inf or a singular denominator.
// Workspace: s.pade[0..7]; A is read from s.pade[7] and F is left in s.pade[0].
__device__ bool expm_dev(Shared &s) {
    double *A = s.pade[7];
    double *B = s.pade[0], *B2 = s.pade[1], *B4 = s.pade[2], *B6 = s.pade[3], *Tm = s.pade[4], *U = s.pade[5],
           *V = s.pade[6];
    __shared__ double norm1;
    __shared__ int sq;
    if (threadIdx.x == 0) {
        double nm = 0.0;
        for (int j = 0; j < MP2; ++j) {
            double c = 0.0;
            for (int i = 0; i < MP2; ++i) c += fabs(A[i + j * MP2]);
            nm = fmax(nm, c);
        }
        norm1 = nm;
        const double theta13 = 5.371920351148152;
        sq = (isfinite(nm) && nm > theta13) ? (int)ceil(log2(nm / theta13)) : 0;
    }
    __syncthreads();
    if (!isfinite(norm1)) return false;
    double c[14];
    c[0] = 1.0;
#pragma unroll
    for (int j = 0; j < 13; ++j) c[j + 1] = c[j] * (double)(13 - j) / ((double)(j + 1) * (double)(26 - j));
    const double scale = ldexp(1.0, -sq);
    for (int e = threadIdx.x; e < MP2 * MP2; e += T) B[e] = A[e] * scale;
    __syncthreads();
    mm(B, B, B2);
    mm(B2, B2, B4);
    mm(B4, B2, B6);
    for (int e = threadIdx.x; e < MP2 * MP2; e += T) Tm[e] = c[13] * B6[e] + c[11] * B4[e] + c[9] * B2[e];
    __syncthreads();
    mm(B6, Tm, A);  // A is free now: W = B6 (c13 B6 + c11 B4 + c9 B2)
    for (int e = threadIdx.x; e < MP2 * MP2; e += T) {
        A[e] += c[7] * B6[e] + c[5] * B4[e] + c[3] * B2[e];
        if (e % MP2 == e / MP2) A[e] += c[1];
    }
    __syncthreads();
    mm(B, A, U);  // U = B W
    for (int e = threadIdx.x; e < MP2 * MP2; e += T) Tm[e] = c[12] * B6[e] + c[10] * B4[e] + c[8] * B2[e];
    __syncthreads();
    mm(B6, Tm, V);
    for (int e = threadIdx.x; e < MP2 * MP2; e += T) {
        double vv = V[e] + c[6] * B6[e] + c[4] * B4[e] + c[2] * B2[e];
        if (e % MP2 == e / MP2) vv += c[0];
        const double u = U[e];
        B2[e] = vv - u;  // P = V - U
        B4[e] = vv + u;  // Q = V + U (becomes the solution)
    }
    __syncthreads();
    // LU with partial pivoting of P (B2), applied to Q (B4): one column per step.
    double *P = B2, *Q = B4;
    __shared__ int singular;
    if (threadIdx.x == 0) singular = 0;
    __syncthreads();
    for (int col = 0; col < MP2; ++col) {
        if (threadIdx.x == 0) {
            int p = col;
            double best = fabs(P[col + col * MP2]);
            for (int i = col + 1; i < MP2; ++i) {
                const double vv = fabs(P[i + col * MP2]);
                if (vv > best) {
                    best = vv;
                    p = i;
                }
            }
            s.piv[col] = p;
            if (best == 0.0) singular = 1;
        }
        __syncthreads();
        if (singular) return false;
        const int p = s.piv[col];
        if (p != col)
            for (int j = threadIdx.x; j < MP2; j += T) {
                double t0 = P[col + j * MP2];
                P[col + j * MP2] = P[p + j * MP2];
                P[p + j * MP2] = t0;
                t0 = Q[col + j * MP2];
                Q[col + j * MP2] = Q[p + j * MP2];
                Q[p + j * MP2] = t0;
            }
        __syncthreads();
        const double inv = 1.0 / P[col + col * MP2];
        // eliminate below the pivot in P (columns > col) and in every column of Q
        for (int e = threadIdx.x; e < (MP2 - col - 1) * (2 * MP2); e += T) {
            const int i = col + 1 + e % (MP2 - col - 1);
            const int j = e / (MP2 - col - 1);
            const double l = P[i + col * MP2] * inv;
            if (j < MP2) {
                if (j > col) P[i + j * MP2] -= l * P[col + j * MP2];
            } else {
                Q[i + (j - MP2) * MP2] -= l * Q[col + (j - MP2) * MP2];
            }
        }
        __syncthreads();
        for (int i = col + 1 + threadIdx.x; i < MP2; i += T) P[i + col * MP2] *= inv;
        __syncthreads();
    }
    // back substitution, one column of Q per thread group
    for (int j = threadIdx.x; j < MP2; j += T) {
        double *q = Q + j * MP2;
        for (int c2 = MP2 - 1; c2 >= 0; --c2) {
            q[c2] /= P[c2 + c2 * MP2];
            for (int i = 0; i < c2; ++i) q[i] -= P[i + c2 * MP2] * q[c2];
        }
    }
    __syncthreads();
    double *R = Q, *Tmp = B6;
    for (int k = 0; k < sq; ++k) {
        mm(R, R, Tmp);
        double *t0 = R;
        R = Tmp;
        Tmp = t0;
    }
    for (int e = threadIdx.x; e < MP2 * MP2; e += T) s.pade[0][e] = R[e];
    __syncthreads();
    __shared__ int bad;
    if (threadIdx.x == 0) {
        bad = 0;
        for (int e = 0; e < MP2 * MP2; ++e)
            if (!isfinite(s.pade[0][e])) bad = 1;
    }
    __syncthreads();
    return !bad;
}

__device__ __forceinline__ double round2(double t) {
    const double sc = pow(10.0, floor(log10(t)) - 1.0);
    return ceil(t / sc) * sc;
}

// ---- one instance --------------------------------------------------------------------------
__device__ void solve_instance(const CufspBatchArgs &a, cg::cluster_group &cl, Shared &s, double *__restrict__ W,
                               int &buf) {
    const int n = s.in.n;
    const int nb = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const int chunk = ((n + nb - 1) / nb + 31) & ~31;
    const int i0 = min(n, rank * chunk), i1 = min(n, i0 + chunk);
    double *v = a.p + s.in.off;
    const double *tab = a.tables + s.in.tab;
    auto vec = [&](int k) -> double * { return k == 0 ? v : W + (size_t)(k - 1) * n; };
    const double delta = 1.2, gamma = 0.9;
    double t_now = 0.0, t_new = 0.0, xm = 1.0 / M, err_loc = 0.0;
    const double btol = a.anorm * a.tol;
    int steps = 0, rejects = 0, matvecs = 0, status = 0;
    Regs g;
    load_regs(s.in, g);

    while (t_now < a.t_final && status == 0) {
        if (steps >= a.max_steps) {
            status = 1;
            break;
        }
        // beta = ||v||
        double acc1 = 0.0;
        for (int i = i0 + (int)threadIdx.x; i < i1; i += T) acc1 = fma(v[i], v[i], acc1);
        cluster_sum1(cl, s, acc1, buf);
        const double beta = sqrt(s.tot[0]);
        if (!isfinite(beta)) {
            status = 2;
            break;
        }
        if (beta == 0.0) {  // exp(tA) 0 = 0
            t_now = a.t_final;
            break;
        }
        for (int e = threadIdx.x; e < MP2 * MP2; e += T) s.H[e] = 0.0;
        for (int e = threadIdx.x; e < MP2; e += T) s.rho[e] = 0.0;
        __syncthreads();
        if (threadIdx.x == 0) s.rho[0] = 1.0 / beta;
        __syncthreads();
        if (steps == 0) {  // first-step size (src/KryExpvFSP.cu:45-51)
            const double fact = pow((M + 1) / exp(1.0), M + 1) * sqrt(2.0 * 3.14159265358979323846 * (M + 1));
            t_new = (1.0 / a.anorm) * pow((fact * a.tol) / (4.0 * beta * a.anorm), 1.0 / M);
        }
        // Arnoldi
        int mb = M, k1 = 2;
        double avnorm = 0.0;
        for (int j = 0; j < M; ++j) {
            const int istart = IOP ? max(0, j - QIOP + 1) : 0;
            const int K = j - istart + 1;
            const double *vj = vec(j);
            double *w = vec(j + 1);
            const double rj = s.rho[j];
            // generator action (own chunk; neighbours read anywhere in the instance)
            for (int i = i0 + (int)threadIdx.x; i < i1; i += T) w[i] = apply_at(g, tab, vj, i, rj);
            // Gram-Schmidt dots in groups of 8 (each thread re-reads only its own w entries)
            for (int k0 = 0; k0 < K; k0 += 8) {
                double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                const double *vb[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) vb[k] = vec(istart + min(k0 + k, K - 1));
                if (K - k0 >= 8) {
                    for (int i = i0 + (int)threadIdx.x; i < i1; i += T) {
                        const double wi = w[i];
#pragma unroll
                        for (int k = 0; k < 8; ++k) acc[k] = fma(vb[k][i], wi, acc[k]);
                    }
                } else {
                    for (int i = i0 + (int)threadIdx.x; i < i1; i += T) {
                        const double wi = w[i];
#pragma unroll
                        for (int k = 0; k < 8; ++k)
                            if (k0 + k < K) acc[k] = fma(vb[k][i], wi, acc[k]);
                    }
                }
                warp_partials8(s, acc, k0, K);
            }
            cluster_finish(cl, s, K, buf);
            for (int k = threadIdx.x; k < K; k += T) {
                const double h = s.rho[istart + k] * s.tot[k];
                s.H[(istart + k) + j * MP2] = h;
                s.gam[istart + k] = h * s.rho[istart + k];
            }
            __syncthreads();
            double acc2 = 0.0;
            for (int i = i0 + (int)threadIdx.x; i < i1; i += T) {
                double wi = w[i];
                int k = 0;
                for (; k + 4 <= K; k += 4) {
                    wi = fma(-s.gam[istart + k], vec(istart + k)[i], wi);
                    wi = fma(-s.gam[istart + k + 1], vec(istart + k + 1)[i], wi);
                    wi = fma(-s.gam[istart + k + 2], vec(istart + k + 2)[i], wi);
                    wi = fma(-s.gam[istart + k + 3], vec(istart + k + 3)[i], wi);
                }
                for (; k < K; ++k) wi = fma(-s.gam[istart + k], vec(istart + k)[i], wi);
                w[i] = wi;
                acc2 = fma(wi, wi, acc2);
            }
            cluster_sum1(cl, s, acc2, buf);
            const double sn = sqrt(s.tot[0]);
            ++matvecs;
            if (!isfinite(sn)) {
                status = 2;
                break;
            }
            // happy breakdown (src/KryExpvFSP.cu:90-98) with the threshold divided by the remaining time
            // (when above 1): the jump to t_final then stays within tol
            if (sn < btol / fmax(1.0, a.t_final - t_now)) {
                k1 = 0;
                mb = j + 1;
                break;
            }
            if (threadIdx.x == 0) {
                s.H[(j + 1) + j * MP2] = sn;
                s.rho[j + 1] = 1.0 / sn;
            }
            __syncthreads();
        }
        if (status) break;
        double tau = fmin(a.t_final - t_now, t_new);
        if (k1 == 0) {
            tau = a.t_final - t_now;
        } else {  // avnorm = ||A v_m|| (src/KryExpvFSP.cu:114-120)
            const double *vm = vec(M);
            const double rm = s.rho[M];
            double acc3 = 0.0;
            for (int i = i0 + (int)threadIdx.x; i < i1; i += T) {
                const double r = apply_at(g, tab, vm, i, rm);
                acc3 = fma(r, r, acc3);
            }
            cluster_sum1(cl, s, acc3, buf);
            avnorm = sqrt(s.tot[0]);
            ++matvecs;
            if (!isfinite(avnorm)) {
                status = 2;
                break;
            }
            if (threadIdx.x == 0) s.H[(M + 1) + M * MP2] = 1.0;
            __syncthreads();
        }
        // rejection loop (src/KryExpvFSP.cu:122-158)
        bool accepted = false;
        int mx = mb + k1;
        while (rejects <= a.max_reject) {
            for (int e = threadIdx.x; e < MP2 * MP2; e += T) s.pade[7][e] = tau * s.H[e];
            __syncthreads();
            if (!expm_dev(s)) {
                status = 2;
                break;
            }
            const double *F = s.pade[0];
            if (k1 == 0) {
                err_loc = btol;
                accepted = true;
                break;
            }
            const double phi1 = fabs(beta * F[mx - 2]);
            const double phi2 = fabs(beta * F[mx - 1] * avnorm);
            if (phi1 > phi2 * 10.0) {
                err_loc = phi2;
                xm = 1.0 / (double)mx;
            } else if (phi1 > phi2) {
                err_loc = (phi1 * phi2) / (phi1 - phi2);
                xm = 1.0 / (double)mx;
            } else {
                err_loc = phi1;
                xm = 1.0 / (double)(mx - 1);
            }
            if (!isfinite(err_loc)) {
                status = 2;
                break;
            }
            if (err_loc <= delta * tau * a.tol) {
                accepted = true;
                break;
            }
            tau = round2(gamma * tau * pow(tau * a.tol / err_loc, xm));
            ++rejects;
        }
        if (status) break;
        if (!accepted) {
            status = 1;
            break;
        }
        // v = beta V[:, 0:mx] F(0:mx, 0) = sum_k (beta F_k0 rho_k) W_k
        mx = mb + max(0, k1 - 1);
        for (int k = threadIdx.x; k < mx; k += T) s.coefc[k] = beta * s.pade[0][k] * s.rho[k];
        __syncthreads();
        for (int i = i0 + (int)threadIdx.x; i < i1; i += T) {
            double r = 0.0;
            for (int k = 0; k < mx; ++k) r = fma(s.coefc[k], vec(k)[i], r);
            v[i] = r;
        }
        const bool last = tau >= a.t_final - t_now;
        t_now = last ? a.t_final : t_now + tau;
        if (err_loc > 0.0) t_new = round2(gamma * tau * pow(tau * a.tol / err_loc, xm));
        if (!(t_new > 0.0) || !isfinite(t_new)) t_new = a.t_final - t_now;
        ++steps;
        cl.sync();  // v complete before the next step's generator action reads it
    }
    if (rank == 0 && threadIdx.x == 0) {
        CufspBatchStat st;
        st.t = t_now;
        st.err = err_loc;
        st.steps = steps;
        st.rejects = rejects;
        st.matvecs = matvecs;
        st.status = status;
        a.stats[s.inst_idx] = st;
    }
}

}  // namespace cufsp_batch

// Dynamic shared memory the kernel needs (read by the host after loading).
extern "C" __device__ const int cufsp_batch_smem_bytes = (int)sizeof(cufsp_batch::Shared);

extern "C" __global__ void __launch_bounds__(CUFSP_BATCH_THREADS, CUFSP_BATCH_MINB)
    cufsp_batch_expv(const CufspBatchArgs a) {
    using namespace cufsp_batch;
    extern __shared__ __align__(16) unsigned char dsm[];
    Shared &s = *reinterpret_cast<Shared *>(dsm);
    cg::cluster_group cl = cg::this_cluster();
    const int nb = (int)cl.num_blocks();
    const int cid = (int)(blockIdx.x / nb);
    double *W = a.work + (size_t)cid * (size_t)a.work_stride;
    int buf = 0;
    for (int it = 0; it < a.n_inst; ++it) {  // at most one instance per iteration and cluster
        if (cl.block_rank() == 0 && threadIdx.x == 0) s.inst_idx = (int)atomicAdd(a.counter, 1u);
        cl.sync();
        if (threadIdx.x == 0) s.inst_idx = *cl.map_shared_rank(&s.inst_idx, 0);
        cl.sync();  // every CTA has read rank 0's index before rank 0 can overwrite it
        if (s.inst_idx >= a.n_inst) break;
        const int idx = a.order[s.inst_idx];
        if (threadIdx.x == 0) s.inst_idx = idx;
        for (int e = threadIdx.x; e < (int)(sizeof(CufspBatchInst) / sizeof(int)); e += T)
            reinterpret_cast<int *>(&s.in)[e] = reinterpret_cast<const int *>(a.inst + idx)[e];
        __syncthreads();
        solve_instance(a, cl, s, W, buf);
        cl.sync();  // the cluster's workspace is free again
    }
}

#endif  // __CUDACC_RTC__
#endif  // CUFSP_BATCH_CUH
