// cufsp_kron_rtc.cuh -- KRONECKER generator action specialised per network and box, for the networks
// the plane kernel (cufsp_plane.cuh) does not take: more than 3 species, changes larger than one
// molecule, odd or long species-0 extents.
//
// Same operator as k_kron_mv (cufsp_kron.cu) and the reference's fspmat_sdkron_mv
// (src/fspmat_kron_kernels.cu:51-129):
//   y[i] (+)= alpha * sum_r c_r ( a_r(x_i - nu_r) x[i - d_r] 1{x_i - nu_r in box} - a_r(x_i) x[i] ),
//   a_r(x) = prod_s f_{r,s}(x_s),
// with the propensities computed from the factor tables as the states are visited (matrix-free: the
// only vectors read are x, at the state and at the reaction sources, and y).
//
// Compiled by NVRTC when a KRONECKER generator is created, after a prefix (cufsp_kron.cu) that fixes
// the box, the stoichiometry and the kind of every factor as constants: 0 a table of ones (no
// work), 1 the identity f(x) = x (no lookup), 2 a tabulated function, read from shared memory where
// the CTA stages the tables it needs (through L1 when they exceed 40 KB).  Each thread owns one aligned pair of states (i, i + 1), i
// even: x[i..i+1] and y[i..i+1] are 16-byte accesses, and the sources of a reaction with an even
// shift d_r are one 16-byte load (two 8-byte loads for an odd shift).  The gathers of a chunk of
// reactions are issued before their first use.  The transposed operator (adjoint solves) is the same
// pass with the propensity at the state and the gather at x + nu_r.
#ifndef CUFSP_KRON_RTC_CUH
#define CUFSP_KRON_RTC_CUH

struct CufspKronRtcArgs {
    const double *tables;   // packed tabulated factors (kind 2 only), t_off(r, s) + x
    const double *d_alpha;  // nullable device scalar multiplying every coefficient
    const int *d_skip;      // nullable: return at once when *d_skip != 0
    long long i_begin, i_end;
    double coef[CUFSP_KRON_RTC_MAX_R];  // alpha * c_r
};

#ifdef __CUDACC_RTC__

namespace cufsp_kron {

constexpr int NS = CUFSP_KRON_NS;
constexpr int NR = CUFSP_KRON_NR;
constexpr long long N = CUFSP_KRON_N;
constexpr int TS = CUFSP_KRON_TS;  // doubles of packed tables (>= 1)
constexpr int CHUNK = CUFSP_KRON_CHUNK;

// The generated prefix defines, in this namespace, constexpr functions of constant indices:
//   ext(s), nu(r, s), shift(r), kind(r, s) (0 ones, 1 identity, 2 table), t_off(r, s) (packed offset)

struct State {
    int x[NS];
};

__device__ __forceinline__ State decode(unsigned i) {
    State st;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        if (s == NS - 1) {
            st.x[s] = (int)i;
        } else {
            const unsigned q = i / (unsigned)ext(s);
            st.x[s] = (int)(i - q * (unsigned)ext(s));
            i = q;
        }
    }
    return st;
}

__device__ __forceinline__ long long clamp_index(long long j) { return j < 0 ? 0 : (j > N - 1 ? N - 1 : j); }

// f_{R,s}(v) for a factor of kind 1 (identity) or 2 (table); kind 0 (ones) never reaches here.
template <int R>
__device__ __forceinline__ double factor(const double *tab, int s, int v) {
    return kind(R, s) == 1 ? (double)v : tab[t_off(R, s) + v];
}

// a_r at the state (diag) and at its source x - nu_r (src, 0 outside the box).
template <int R>
__device__ __forceinline__ void propensities(const double *tab, const State &st, double &diag, double &src) {
    double d = 1.0, sv = 1.0;
    bool ok = true;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int v = st.x[s];
        if (nu(R, s) != 0) {
            int w = v - nu(R, s);
            ok = ok && w >= 0 && w < ext(s);
            w = w < 0 ? 0 : (w >= ext(s) ? ext(s) - 1 : w);  // in-bounds lookup; the product is dropped
            if (kind(R, s) != 0) {
                d *= factor<R>(tab, s, v);
                sv *= factor<R>(tab, s, w);
            }
        } else if (kind(R, s) != 0) {
            const double f = factor<R>(tab, s, v);
            d *= f;
            sv *= f;
        }
    }
    diag = d;
    src = ok ? sv : 0.0;
}

// Transposed generator (adjoint solves): (A^T l)(x) = sum_r c_r a_r(x) (l[x + nu_r] 1{x + nu_r in box}
// - l[x]): the propensity at the state, the gather at x + nu_r.
template <int R>
__device__ __forceinline__ void propensities_t(const double *tab, const State &st, double &diag, double &dst) {
    double d = 1.0;
    bool ok = true;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int v = st.x[s];
        if (nu(R, s) != 0) {
            const int w = v + nu(R, s);
            ok = ok && w >= 0 && w < ext(s);
        }
        if (kind(R, s) != 0) d *= factor<R>(tab, s, v);
    }
    diag = d;
    dst = ok ? d : 0.0;
}

struct Pending {
    double xs0, xs1;  // x at the two sources
};

template <int R, bool TRANS>
__device__ __forceinline__ void load_reaction(const double *__restrict__ x, long long i, bool pair, Pending &q) {
    constexpr long long D = TRANS ? -shift(R) : shift(R);
    const long long s0 = clamp_index(i - D), s1 = clamp_index(i + 1 - D);
    if constexpr ((D & 1) == 0) {
        if (pair && s1 == s0 + 1) {  // sources of an even shift are an aligned pair
            const double2 xv = __ldg(reinterpret_cast<const double2 *>(x + s0));
            q.xs0 = xv.x;
            q.xs1 = xv.y;
            return;
        }
    }
    q.xs0 = __ldg(x + s0);
    q.xs1 = pair ? __ldg(x + s1) : 0.0;
}

template <int R0, int R, bool TRANS>
__device__ __forceinline__ void load_chunk(const double *__restrict__ x, long long i, bool pair, Pending (&q)[CHUNK]) {
    if constexpr (R < NR && R < R0 + CHUNK) {
        load_reaction<R, TRANS>(x, i, pair, q[R - R0]);
        load_chunk<R0, R + 1, TRANS>(x, i, pair, q);
    }
}

template <int R0, int R, bool TRANS>
__device__ __forceinline__ void accumulate_chunk(const CufspKronRtcArgs &a, const double *tab, const State &s0,
                                                 const State &s1, const Pending (&q)[CHUNK], double (&d)[2],
                                                 double (&o)[2]) {
    if constexpr (R < NR && R < R0 + CHUNK) {
        const double c = a.coef[R];
        double d0, f0, d1, f1;
        if constexpr (TRANS) {
            propensities_t<R>(tab, s0, d0, f0);
            propensities_t<R>(tab, s1, d1, f1);
        } else {
            propensities<R>(tab, s0, d0, f0);
            propensities<R>(tab, s1, d1, f1);
        }
        d[0] = fma(c, d0, d[0]);
        d[1] = fma(c, d1, d[1]);
        o[0] = fma(c, f0 * q[R - R0].xs0, o[0]);
        o[1] = fma(c, f1 * q[R - R0].xs1, o[1]);
        accumulate_chunk<R0, R + 1, TRANS>(a, tab, s0, s1, q, d, o);
    }
}

template <int R0, bool TRANS>
__device__ __forceinline__ void all_reactions(const CufspKronRtcArgs &a, const double *tab,
                                              const double *__restrict__ x, long long i, bool pair, const State &s0,
                                              const State &s1, double (&d)[2], double (&o)[2]) {
    if constexpr (R0 < NR) {
        Pending q[CHUNK];
        load_chunk<R0, R0, TRANS>(x, i, pair, q);
        accumulate_chunk<R0, R0, TRANS>(a, tab, s0, s1, q, d, o);
        all_reactions<R0 + CHUNK, TRANS>(a, tab, x, i, pair, s0, s1, d, o);
    }
}

template <bool ACCUM, bool TRANS>
__device__ __forceinline__ void kron_mv(const CufspKronRtcArgs &a, const double *__restrict__ x, double *__restrict__ y) {
#if CUFSP_KRON_TAB_SMEM
    __shared__ double tab[TS];
    if (a.d_skip && *a.d_skip) return;
    for (int k = threadIdx.x; k < TS; k += blockDim.x) tab[k] = __ldg(a.tables + k);
    __syncthreads();
#else
    // tables too large for static shared memory are read through the L1 cache
    const double *__restrict__ tab = a.tables;
    if (a.d_skip && *a.d_skip) return;
#endif
    const double alpha = a.d_alpha ? __ldg(a.d_alpha) : 1.0;
    const long long first = a.i_begin & ~1LL;
    const long long pairs = (a.i_end - first + 1) >> 1;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < pairs;
         k += (long long)gridDim.x * blockDim.x) {
        const long long i = first + 2 * k;
        const bool pair = i + 1 < N;  // the last state of an odd-length vector is alone
        double2 xv, yv = make_double2(0.0, 0.0);
        if (pair) {
            xv = __ldg(reinterpret_cast<const double2 *>(x + i));
            if (ACCUM) yv = *reinterpret_cast<const double2 *>(y + i);
        } else {
            xv = make_double2(__ldg(x + i), 0.0);
            if (ACCUM) yv.x = y[i];
        }
        const State s0 = decode((unsigned)i);
        const State s1 = decode((unsigned)(pair ? i + 1 : i));
        double d[2] = {0.0, 0.0}, o[2] = {0.0, 0.0};
        all_reactions<0, TRANS>(a, tab, x, i, pair, s0, s1, d, o);
        double r0 = alpha * fma(-d[0], xv.x, o[0]);
        double r1 = alpha * fma(-d[1], xv.y, o[1]);
        if (ACCUM) {
            r0 += yv.x;
            r1 += yv.y;
        }
        const bool w0 = i >= a.i_begin, w1 = pair && i + 1 < a.i_end;
        if (w0 && w1) {
            __stcs(reinterpret_cast<double2 *>(y + i), make_double2(r0, r1));
        } else {
            if (w0) y[i] = r0;
            if (w1) y[i + 1] = r1;
        }
    }
}

}  // namespace cufsp_kron

extern "C" __global__ void __launch_bounds__(256, CUFSP_KRON_MINB) cufsp_kron_mv_accum(const CufspKronRtcArgs a,
                                                                                      const double *__restrict__ x,
                                                                                      double *__restrict__ y) {
    cufsp_kron::kron_mv<true, false>(a, x, y);
}

extern "C" __global__ void __launch_bounds__(256, CUFSP_KRON_MINB) cufsp_kron_mv_set(const CufspKronRtcArgs a,
                                                                                    const double *__restrict__ x,
                                                                                    double *__restrict__ y) {
    cufsp_kron::kron_mv<false, false>(a, x, y);
}

// y = alpha * A^T x (overwrite): the adjoint solves' operator.
extern "C" __global__ void __launch_bounds__(256, CUFSP_KRON_MINB) cufsp_kron_mvT_set(const CufspKronRtcArgs a,
                                                                                     const double *__restrict__ x,
                                                                                     double *__restrict__ y) {
    cufsp_kron::kron_mv<false, true>(a, x, y);
}

#endif  // __CUDACC_RTC__
#endif  // CUFSP_KRON_RTC_CUH
