// cufsp_sparse_rtc.cuh -- sparse-format generator action specialised per network and box.
//
// Same operator as k_sparse_mv (cufsp_sparse.cu), the stand-in for the reference's CSR/HYB actions
// (src/fspmat_csr_kernels.cu:123-136, src/fspmat_hyb_kernels.cu:66-106):
//   y[i] (+)= alpha * sum_r c_r ( P_r[i - d_r] x[i - d_r] 1{x_i - nu_r in box} - P_r[i] x[i] ),
// with the propensity table P_r[i] = a_r(x_i) stored reaction-major.
//
// Compiled by NVRTC when a CSR/HYB generator is created, after a prefix (cufsp_sparse.cu) that fixes
// the box and every reaction's stoichiometry as constants: divisions by the species extents become
// multiplications, the validity test of each reaction touches only the species it changes, and the
// reaction loop is unrolled with every shift d_r a literal.
//
// Each thread owns one aligned pair of states (i, i + 1), i even: x[i..i+1], y[i..i+1] and every
// P_r[i..i+1] are single 16-byte loads; the shifted source pair (i - d_r, i + 1 - d_r) is one 16-byte
// load of P_r and one of x when d_r is even, two 8-byte loads each when it is odd.  All loads of a
// pair are issued before the first use (memory-level parallelism), and the table rows use the
// default L2 policy, so that the shifted re-read of a row -- by the CTA |d_r| states away -- hits L2
// instead of DRAM; y is written with the streaming policy.
#ifndef CUFSP_SPARSE_RTC_CUH
#define CUFSP_SPARSE_RTC_CUH

struct CufspSparseRtcArgs {
    const double *P;        // [NR][n] propensity table
    const double *d_alpha;  // nullable device scalar multiplying every coefficient
    const int *d_skip;      // nullable: return at once when *d_skip != 0
    long long i_begin, i_end;
    double coef[CUFSP_SPARSE_RTC_MAX_R];  // alpha * c_r
};

#ifdef __CUDACC_RTC__

namespace cufsp_sparse {

constexpr int NS = CUFSP_SPARSE_NS;
constexpr int NR = CUFSP_SPARSE_NR;
constexpr long long N = CUFSP_SPARSE_N;

// The generated prefix defines, in this namespace, constexpr functions of a constant index:
//   ext(s)       extent b_s + 1 of species s
//   nu(r, s)     net change of species s when reaction r fires
//   shift(r)     d_r = sum_s nu(r, s) * stride_s
//   touches(r, s) nu(r, s) != 0

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

template <int R>
__device__ __forceinline__ bool source_in_box(const State &st) {
    bool ok = true;
#pragma unroll
    for (int s = 0; s < NS; ++s)
        if (touches(R, s)) {
            const int v = st.x[s] - nu(R, s);
            ok = ok && v >= 0 && v < ext(s);
        }
    return ok;
}

__device__ __forceinline__ long long clamp_index(long long j) { return j < 0 ? 0 : (j > N - 1 ? N - 1 : j); }

// Loads of one reaction for the pair (i, i + 1).
struct Pending {
    double2 p;       // P_r[i], P_r[i + 1]
    double ps0, ps1; // P_r at the two sources
    double xs0, xs1; // x at the two sources
};

template <int R>
__device__ __forceinline__ void load_reaction(const double *__restrict__ P, const double *__restrict__ x, long long i,
                                              bool pair, Pending &q) {
    const double *Pr = P + (long long)R * N;
    constexpr long long D = shift(R);
    if (pair) q.p = __ldg(reinterpret_cast<const double2 *>(Pr + i));
    else q.p = make_double2(__ldg(Pr + i), 0.0);
    const long long s0 = clamp_index(i - D), s1 = clamp_index(i + 1 - D);
    if constexpr ((D & 1) == 0) {
        // sources of an even shift are an aligned pair (clamped ends stay aligned: N - 1 is odd only
        // when N is even, and then s0 = N - 2 is even)
        if (pair && s1 == s0 + 1) {
            const double2 pv = __ldg(reinterpret_cast<const double2 *>(Pr + s0));
            const double2 xv = __ldg(reinterpret_cast<const double2 *>(x + s0));
            q.ps0 = pv.x;
            q.ps1 = pv.y;
            q.xs0 = xv.x;
            q.xs1 = xv.y;
            return;
        }
    }
    q.ps0 = __ldg(Pr + s0);
    q.xs0 = __ldg(x + s0);
    q.ps1 = pair ? __ldg(Pr + s1) : 0.0;
    q.xs1 = pair ? __ldg(x + s1) : 0.0;
}

// Reactions are processed in chunks of CHUNK: the loads of a whole chunk are in flight together.
constexpr int CHUNK = CUFSP_SPARSE_CHUNK;

template <int R0, int R>
__device__ __forceinline__ void load_chunk(const double *__restrict__ P, const double *__restrict__ x, long long i,
                                           bool pair, Pending (&q)[CHUNK]) {
    if constexpr (R < NR && R < R0 + CHUNK) {
        load_reaction<R>(P, x, i, pair, q[R - R0]);
        load_chunk<R0, R + 1>(P, x, i, pair, q);
    }
}

template <int R0, int R>
__device__ __forceinline__ void accumulate_chunk(const CufspSparseRtcArgs &a, const State &s0, const State &s1,
                                                 const Pending (&q)[CHUNK], double (&d)[2], double (&o)[2]) {
    if constexpr (R < NR && R < R0 + CHUNK) {
        const double c = a.coef[R];
        d[0] = fma(c, q[R - R0].p.x, d[0]);
        d[1] = fma(c, q[R - R0].p.y, d[1]);
        const double f0 = source_in_box<R>(s0) ? q[R - R0].ps0 * q[R - R0].xs0 : 0.0;
        const double f1 = source_in_box<R>(s1) ? q[R - R0].ps1 * q[R - R0].xs1 : 0.0;
        o[0] = fma(c, f0, o[0]);
        o[1] = fma(c, f1, o[1]);
        accumulate_chunk<R0, R + 1>(a, s0, s1, q, d, o);
    }
}

template <int R0>
__device__ __forceinline__ void all_reactions(const CufspSparseRtcArgs &a, const double *__restrict__ x, long long i,
                                              bool pair, const State &s0, const State &s1, double (&d)[2],
                                              double (&o)[2]) {
    if constexpr (R0 < NR) {
        Pending q[CHUNK];
        load_chunk<R0, R0>(a.P, x, i, pair, q);
        accumulate_chunk<R0, R0>(a, s0, s1, q, d, o);
        all_reactions<R0 + CHUNK>(a, x, i, pair, s0, s1, d, o);
    }
}

template <bool ACCUM>
__device__ __forceinline__ void sparse_mv(const CufspSparseRtcArgs &a, const double *__restrict__ x,
                                          double *__restrict__ y) {
    if (a.d_skip && *a.d_skip) return;
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
        all_reactions<0>(a, x, i, pair, s0, s1, d, o);
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

}  // namespace cufsp_sparse

extern "C" __global__ void __launch_bounds__(256, CUFSP_SPARSE_MINB) cufsp_sparse_mv_accum(const CufspSparseRtcArgs a,
                                                                        const double *__restrict__ x,
                                                                        double *__restrict__ y) {
    cufsp_sparse::sparse_mv<true>(a, x, y);
}

extern "C" __global__ void __launch_bounds__(256, CUFSP_SPARSE_MINB) cufsp_sparse_mv_set(const CufspSparseRtcArgs a,
                                                                      const double *__restrict__ x,
                                                                      double *__restrict__ y) {
    cufsp_sparse::sparse_mv<false>(a, x, y);
}

#endif  // __CUDACC_RTC__
#endif  // CUFSP_SPARSE_RTC_CUH
