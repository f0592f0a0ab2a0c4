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
    long long q_begin, q_end;  // row range of the row and slab kernels
    int *err;                  // watchdog word of the slab kernels (set when a bounded wait expired)
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

// ---- Row kernels: inner factors fixed per lane ------------------------------------------------
// The state index is split i = q * LEN + p: p covers the inner species 0 .. KI-1 (LEN positions), the
// row q the outer species KI .. NS-1.  A warp owns VP * 32 positions of one row chunk, lane-contiguous
// (p = chunk * 32 VP + v * 32 + lane), and sweeps the rows of its chunk; every gather x[i - d_r] is
// then one 256-byte warp access.  The inner factor products of a lane's positions, already multiplied
// by alpha * c_r, are computed once per chunk into registers:
//   A_r(p) = alpha c_r prod_{s<KI} f_{r,s}(p_s - nu_{r,s}) 1{inner source in box}
//   D0(p)  = sum over reactions whose outer factors are all ones of alpha c_r prod_{s<KI} f_{r,s}(p_s)
//   E_r(p) = alpha c_r prod_{s<KI} f_{r,s}(p_s) for the other reactions,
// and the outer factors once per row: G_r(q) (source, 0 outside the box) and Gd_r(q) (state), both
// the constant 1 -- folded away at compile time -- for reactions that leave the outer species alone.
// Per state and reaction the work is one gather and one or two FP64 operations:
//   y[i] (+)= sum_r A_r(p) G_r(q) x[i - d_r] - x[i] (D0(p) + sum_r E_r(p) Gd_r(q)).
// The transposed action takes A_r = alpha c_r prod_{s<KI} f_{r,s}(p_s) 1{inner target in box},
// G_r = prod_{s>=KI} f_{r,s}(q_s) 1{outer target in box} and the gather at x[i + d_r].

namespace cufsp_kron {

constexpr int KI = CUFSP_KRON_K;
constexpr int VP = CUFSP_KRON_V;
constexpr long long LEN = CUFSP_KRON_L;
constexpr long long NCH = (LEN + 32 * VP - 1) / (32 * VP);
constexpr int RC = CUFSP_KRON_RCHUNK;
constexpr int NO = NS - KI > 0 ? NS - KI : 1;  // outer species (array extent)

__device__ __forceinline__ constexpr bool outer_src_one(int r) {
    for (int s = KI; s < NS; ++s)
        if (nu(r, s) != 0 || kind(r, s) != 0) return false;
    return true;
}
__device__ __forceinline__ constexpr bool outer_diag_one(int r) {
    for (int s = KI; s < NS; ++s)
        if (kind(r, s) != 0) return false;
    return true;
}
// Terms: reactions with the same shift whose outer factors are all ones share one gather and one
// per-lane factor (their A_r summed); every other reaction is a term of its own.
__device__ __forceinline__ constexpr int term_owner(int r) {  // first reaction of r's term
    if (!outer_src_one(r)) return r;
    for (int u = 0; u < r; ++u)
        if (outer_src_one(u) && shift(u) == shift(r)) return u;
    return r;
}
__device__ __forceinline__ constexpr int term_of(int r) {  // owners before r's owner
    int t = 0;
    for (int u = 0; u < term_owner(r); ++u) t += term_owner(u) == u ? 1 : 0;
    return t;
}
__device__ __forceinline__ constexpr int n_terms() {
    int t = 0;
    for (int u = 0; u < NR; ++u) t += term_owner(u) == u ? 1 : 0;
    return t;
}
__device__ __forceinline__ constexpr int term_rep(int t) {  // owner reaction of term t
    for (int u = 0; u < NR; ++u)
        if (term_owner(u) == u && term_of(u) == t) return u;
    return 0;
}
constexpr int NT = n_terms();

// Largest and smallest shift d_r (gathers at i - d_r; the transposed pass negates them).
__device__ __forceinline__ constexpr long long shift_max() {
    long long m = 0;
    for (int r = 0; r < NR; ++r) m = shift(r) > m ? shift(r) : m;
    return m;
}
__device__ __forceinline__ constexpr long long shift_min() {
    long long m = 0;
    for (int r = 0; r < NR; ++r) m = shift(r) < m ? shift(r) : m;
    return m;
}

// Factors of reaction R over species [S0, S1) at the multi-index v (indexed from S0): src at v - nu
// (TRANS: at v, with the target v + nu checked), 0 when that leaves the box; diag at v.
template <int R, int S0, int S1, bool TRANS, int M>
__device__ __forceinline__ void span_factors(const double *tab, const int (&v)[M], double &src, double &diag) {
    double d = 1.0, sv = 1.0;
    bool ok = true;
#pragma unroll
    for (int s = S0; s < S1; ++s) {
        const int xs = v[s - S0];
        if (nu(R, s) != 0) {
            int w = TRANS ? xs + nu(R, s) : xs - nu(R, s);
            ok = ok && w >= 0 && w < ext(s);
            if (kind(R, s) != 0) {
                d *= factor<R>(tab, s, xs);
                if (!TRANS) {
                    w = w < 0 ? 0 : (w >= ext(s) ? ext(s) - 1 : w);
                    sv *= factor<R>(tab, s, w);
                }
            }
        } else if (kind(R, s) != 0) {
            const double f = factor<R>(tab, s, xs);
            d *= f;
            sv *= f;
        }
    }
    diag = d;
    src = ok ? (TRANS ? d : sv) : 0.0;
}

template <int V>
struct PosRegs {
    double A[V][NT];  // per term
    double E[V][NR];  // per reaction with outer diagonal factors
    double D0[V];
};
using RowRegs = PosRegs<VP>;

template <int R, bool TRANS, int V>
__device__ __forceinline__ void chunk_prologue(const CufspKronRtcArgs &a, double alpha, const double *tab,
                                               const int (&xi)[KI], int v, PosRegs<V> &g) {
    if constexpr (R < NR) {
        double src, diag;
        span_factors<R, 0, KI, TRANS, KI>(tab, xi, src, diag);
        const double c = alpha * a.coef[R];
        if constexpr (term_owner(R) == R) {
            g.A[v][term_of(R)] = c * src;
        } else {
            g.A[v][term_of(R)] = fma(c, src, g.A[v][term_of(R)]);
        }
        if constexpr (outer_diag_one(R)) {
            g.D0[v] = fma(c, diag, g.D0[v]);
        } else {
            g.E[v][R] = c * diag;
        }
        chunk_prologue<R + 1, TRANS, V>(a, alpha, tab, xi, v, g);
    }
}

template <int R, bool TRANS>
__device__ __forceinline__ void row_words(const double *tab, const int (&z)[NO], double (&G)[NR], double (&Gd)[NR]) {
    if constexpr (R < NR) {
        if constexpr (!outer_src_one(R) || !outer_diag_one(R)) {
            double src, diag;
            span_factors<R, KI, NS, TRANS, NO>(tab, z, src, diag);
            G[R] = src;
            Gd[R] = diag;
        }
        row_words<R + 1, TRANS>(tab, z, G, Gd);
    }
}

// Gathers of terms T0 .. T0 + RC - 1 (the sources of term T at i - d, d the shift of its owner).
template <int T0, int T, bool TRANS, bool SAFE>
__device__ __forceinline__ void rows_load(const double *__restrict__ x, const long long (&i)[VP], double (&q)[RC][VP]) {
    if constexpr (T < NT && T < T0 + RC) {
        constexpr long long D = shift(term_rep(T));
#pragma unroll
        for (int v = 0; v < VP; ++v) {
            long long j = TRANS ? i[v] + D : i[v] - D;
            if (!SAFE) j = clamp_index(j);
            q[T - T0][v] = __ldg(x + j);
        }
        rows_load<T0, T + 1, TRANS, SAFE>(x, i, q);
    }
}

template <int T0, int T>
__device__ __forceinline__ void rows_acc(const RowRegs &g, const double (&G)[NR], const double (&q)[RC][VP],
                                         double (&acc)[VP]) {
    if constexpr (T < NT && T < T0 + RC) {
        constexpr int R = term_rep(T);
#pragma unroll
        for (int v = 0; v < VP; ++v) {
            if constexpr (outer_src_one(R)) {
                acc[v] = fma(g.A[v][T], q[T - T0][v], acc[v]);
            } else {
                acc[v] = fma(g.A[v][T] * G[R], q[T - T0][v], acc[v]);
            }
        }
        rows_acc<T0, T + 1>(g, G, q, acc);
    }
}

template <int T0, bool TRANS, bool SAFE>
__device__ __forceinline__ void rows_all(const double *__restrict__ x, const RowRegs &g, const double (&G)[NR],
                                         const long long (&i)[VP], double (&acc)[VP]) {
    if constexpr (T0 < NT) {
        double q[RC][VP];
        rows_load<T0, T0, TRANS, SAFE>(x, i, q);
        rows_acc<T0, T0>(g, G, q, acc);
        rows_all<T0 + RC, TRANS, SAFE>(x, g, G, i, acc);
    }
}

template <int R, int V>
__device__ __forceinline__ void rows_diag(const PosRegs<V> &g, const double (&Gd)[NR], double (&dg)[V]) {
    if constexpr (R < NR) {
        if constexpr (!outer_diag_one(R)) {
#pragma unroll
            for (int v = 0; v < V; ++v) dg[v] = fma(g.E[v][R], Gd[R], dg[v]);
        }
        rows_diag<R + 1, V>(g, Gd, dg);
    }
}

// Decode inner position p (< LEN) into the inner multi-index.
__device__ __forceinline__ void inner_decode(long long p, int (&xi)[KI]) {
#pragma unroll
    for (int s = 0; s < KI; ++s) {
        const long long qq = p / ext(s);
        xi[s] = (int)(p - qq * ext(s));
        p = qq;
    }
}

// Decode row q into the outer multi-index.
__device__ __forceinline__ void outer_decode(long long q, int (&z)[NO]) {
#pragma unroll
    for (int s = KI; s < NS; ++s) {
        if (s == NS - 1) {
            z[s - KI] = (int)q;
        } else {
            const long long qq = q / ext(s);
            z[s - KI] = (int)(q - qq * ext(s));
            q = qq;
        }
    }
}

template <bool ACCUM, bool TRANS>
__device__ __forceinline__ void kron_rows(const CufspKronRtcArgs &a, const double *__restrict__ x,
                                          double *__restrict__ y) {
    if (a.d_skip && *a.d_skip) return;
    const double *__restrict__ tab = a.tables;
    const double alpha = a.d_alpha ? __ldg(a.d_alpha) : 1.0;
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long total = (a.q_end - a.q_begin) * NCH;
    constexpr long long DMAX = TRANS ? -shift_min() : shift_max();  // largest amount subtracted
    constexpr long long DMIN = TRANS ? -shift_max() : shift_min();
    long long cur = -1;
    RowRegs g;
    long long pos[VP];
    bool act[VP];
    // The chunks of a warp's (row, chunk) pairs repeat with period NCH: when the warp count is a
    // multiple of NCH the prologue runs once.
    for (long long t = gw; t < total; t += nw) {
        const long long ch = t % NCH;
        const long long q = a.q_begin + t / NCH;
        if (ch != cur) {
            cur = ch;
#pragma unroll
            for (int v = 0; v < VP; ++v) {
                pos[v] = ch * (32 * VP) + v * 32 + lane;
                act[v] = pos[v] < LEN;
                long long rem = act[v] ? pos[v] : LEN - 1;
                int xi[KI];
#pragma unroll
                for (int s = 0; s < KI; ++s) {
                    const long long qq = rem / ext(s);
                    xi[s] = (int)(rem - qq * ext(s));
                    rem = qq;
                }
                g.D0[v] = 0.0;
                chunk_prologue<0, TRANS, VP>(a, alpha, tab, xi, v, g);
            }
        }
        int z[NO];
        {
            long long rem = q;
#pragma unroll
            for (int s = KI; s < NS; ++s) {
                if (s == NS - 1) {
                    z[s - KI] = (int)rem;
                } else {
                    const long long qq = rem / ext(s);
                    z[s - KI] = (int)(rem - qq * ext(s));
                    rem = qq;
                }
            }
        }
        double G[NR], Gd[NR];
        row_words<0, TRANS>(tab, z, G, Gd);
        long long i[VP];
        double xv[VP], yv[VP], acc[VP], dg[VP];
#pragma unroll
        for (int v = 0; v < VP; ++v) {
            i[v] = q * LEN + (act[v] ? pos[v] : 0);
            xv[v] = __ldg(x + i[v]);
            yv[v] = (ACCUM && act[v]) ? __ldcs(y + i[v]) : 0.0;
            acc[v] = 0.0;
            dg[v] = g.D0[v];
        }
        const bool safe = q * LEN >= DMAX && (q + 1) * LEN - 1 - DMIN <= N - 1;
        if (safe) {
            rows_all<0, TRANS, true>(x, g, G, i, acc);
        } else {
            rows_all<0, TRANS, false>(x, g, G, i, acc);
        }
        rows_diag<0, VP>(g, Gd, dg);
#pragma unroll
        for (int v = 0; v < VP; ++v) {
            if (act[v]) {
                double r = fma(-dg[v], xv[v], acc[v]);
                if (ACCUM) r += yv[v];
                __stcs(y + i[v], r);
            }
        }
    }
}

}  // namespace cufsp_kron

extern "C" __global__ void __launch_bounds__(256, CUFSP_KRON_ROWS_MINB) cufsp_kron_rows_accum(
    const CufspKronRtcArgs a, const double *__restrict__ x, double *__restrict__ y) {
    cufsp_kron::kron_rows<true, false>(a, x, y);
}

extern "C" __global__ void __launch_bounds__(256, CUFSP_KRON_ROWS_MINB) cufsp_kron_rows_set(
    const CufspKronRtcArgs a, const double *__restrict__ x, double *__restrict__ y) {
    cufsp_kron::kron_rows<false, false>(a, x, y);
}

extern "C" __global__ void __launch_bounds__(256, CUFSP_KRON_ROWS_MINB) cufsp_kron_rowsT_set(
    const CufspKronRtcArgs a, const double *__restrict__ x, double *__restrict__ y) {
    cufsp_kron::kron_rows<false, true>(a, x, y);
}

// ---- Slab kernels: the row kernels' arithmetic on rows staged in shared memory by TMA ----------
// For networks whose reactions move the row index q by at most H rows (|dq| <= H) and whose rows fit
// shared memory: a CTA owns a segment of whole rows [q0, q1) and streams rows q0 - H .. q1 - 1 + H
// through a ring of SS stages, one bulk copy (cp.async.bulk + mbarrier complete_tx) per row of x
// (and of y, for the rows it computes, in the accumulate form), issued by one thread as stages free
// up.  Row q is computed from the stages of rows q - H .. q + H: every gather is a shared-memory load
// at a compile-time offset, and every x value crosses HBM once per segment (plus 2H halo rows).  Each
// staged x row has GD zero guard doubles on both sides, so inner sources outside the row read 0
// (their factor is 0 as well) without a clamp.  Rows outside the box are never copied: their stage
// arrives empty and their outer factor is 0.  Every mbarrier wait is bounded; on expiry the CTA
// drains its copies (bounded), sets the watchdog word and leaves its rows unwritten.

#if CUFSP_KRON_SLAB
namespace cufsp_kron {

constexpr int ST = CUFSP_KRON_SLAB_T;   // threads per CTA
constexpr int VS = CUFSP_KRON_SLAB_VS;  // positions per thread, ST apart
constexpr int SS = CUFSP_KRON_SLAB_S;   // ring stages
constexpr int HB = CUFSP_KRON_SLAB_H;   // row halo on each side
constexpr int GD = CUFSP_KRON_SLAB_G;   // zero guard doubles on each side of a staged x row (even)
constexpr int TW = ST * VS;                          // positions of a CTA's tile of a row
constexpr long long NTILE = (LEN + TW - 1) / TW;     // tiles per row
constexpr int PITCH = TW + 2 * GD;
constexpr int SD = PITCH + TW;                       // stage: guarded x tile, then the y tile
constexpr long long QN = N / LEN;                    // rows in the box
#ifndef CUFSP_KRON_SLAB_WAIT_TRIES
#define CUFSP_KRON_SLAB_WAIT_TRIES (1 << 20)
#endif
#ifndef CUFSP_KRON_SLAB_SHFL
#define CUFSP_KRON_SLAB_SHFL 1
#endif

__device__ __forceinline__ constexpr long long istride(int s) {
    long long st = 1;
    for (int u = 0; u < s; ++u) st *= ext(u);
    return st;
}
__device__ __forceinline__ constexpr long long inner_shift(int r) {
    long long d = 0;
    for (int s = 0; s < KI; ++s) d += (long long)nu(r, s) * istride(s);
    return d;
}
__device__ __forceinline__ constexpr long long row_shift(int r) { return (shift(r) - inner_shift(r)) / LEN; }

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity, int tries) {
    for (int it = 0; it < tries; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tma_load(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Leading species of extent 2 (binary switches) up to lane bit 4: the state index of such a species'
// flip differs from the state's in one bit below 32, i.e. in the lane index (positions are
// lane-contiguous and ST is a multiple of 32).
__device__ __forceinline__ constexpr int binary_prefix() {
    int b = 0;
    while (b < KI && b < 5 && ext(b) == 2) ++b;
    return b;
}
// Mask m when reaction r changes only one binary-prefix species s, by 1, and leaves the row alone: its
// source, wherever its factor is nonzero, is the lane p ^ m (m = 2^s).
__device__ __forceinline__ constexpr int flip_mask(int r) {
    if (!CUFSP_KRON_SLAB_SHFL || row_shift(r) != 0) return 0;
    int m = 0;
    for (int s = 0; s < KI; ++s) {
        if (nu(r, s) == 0) continue;
        if (m != 0 || s >= binary_prefix() || (nu(r, s) != 1 && nu(r, s) != -1)) return 0;
        m = 1 << s;
    }
    return m;
}
// The mask of the term owned by reaction R when every reaction of the term has that same mask (the
// source then comes by a warp shuffle instead of a shared-memory load), else 0.
__device__ __forceinline__ constexpr int xor_mask(int R) {
    const int m = flip_mask(R);
    for (int u = 0; u < NR && m != 0; ++u)
        if (term_owner(u) == R && flip_mask(u) != m) return 0;
    return m;
}

// acc += sum over terms of A_T(p) G_T(q) x[source]; rowp[k] is the staged x row of row q - HB + k.
template <int T, bool TRANS>
__device__ __forceinline__ void slab_terms(const double *const (&rowp)[2 * HB + 1], const PosRegs<VS> &g,
                                           const double (&G)[NR], const int (&lp)[VS], const double (&xv)[VS],
                                           double (&acc)[VS]) {
    if constexpr (T < NT) {
        constexpr int R = term_rep(T);
        constexpr int DQ = TRANS ? -(int)row_shift(R) : (int)row_shift(R);  // source row q - DQ
        constexpr int DP = TRANS ? -(int)inner_shift(R) : (int)inner_shift(R);
        constexpr int XM = xor_mask(R);
        const double *src = rowp[HB - DQ] + (GD - DP);
#pragma unroll
        for (int v = 0; v < VS; ++v) {
            const double xs = XM ? __shfl_xor_sync(0xffffffffu, xv[v], XM) : src[lp[v]];
            if constexpr (outer_src_one(R)) {
                acc[v] = fma(g.A[v][T], xs, acc[v]);
            } else {
                acc[v] = fma(g.A[v][T] * G[R], xs, acc[v]);
            }
        }
        slab_terms<T + 1, TRANS>(rowp, g, G, lp, xv, acc);
    }
}

template <bool ACCUM, bool TRANS>
__device__ __forceinline__ void kron_slab(const CufspKronRtcArgs &a, const double *__restrict__ x,
                                          double *__restrict__ y) {
    extern __shared__ __align__(128) double smem[];
    __shared__ __align__(8) unsigned long long bars[SS];
    __shared__ int failed;
    if (a.d_skip && *a.d_skip) return;
    // CTA = (tile of TW positions, segment of rows); the grid is a multiple of NTILE.
    const long long nrows = a.q_end - a.q_begin;
    const long long nseg = gridDim.x / NTILE;
    const long long tile = blockIdx.x % NTILE, segi = blockIdx.x / NTILE;
    const long long seg = (nrows + nseg - 1) / nseg;
    const long long q0 = a.q_begin + segi * seg;
    const long long q1 = min(a.q_end, q0 + seg);
    const long long p0 = tile * TW;                           // first position of the tile
    const long long xlo = max(0LL, p0 - GD), xhi = min(LEN, p0 + TW + GD);  // staged x positions
    const long long ylen = min(LEN, p0 + TW) - p0;
    if (q0 >= q1) return;  // whole CTA leaves before any barrier or copy
    const int tid = threadIdx.x;
    for (int k = tid; k < SS * SD; k += ST) smem[k] = 0.0;  // guards and never-copied rows stay zero
    if (tid == 0) {
        for (int k = 0; k < SS; ++k) mbar_init(bars + k, 1);
        fence_mbar_init();
        failed = 0;
    }
    fence_proxy_async();
    __syncthreads();

    // Row p >= pbase lives in stage (p - pbase) % SS, phase parity ((p - pbase) / SS) & 1.
    const long long pbase = q0 - HB, plast = q1 - 1 + HB;
    auto stage = [&](long long p) { return smem + ((p - pbase) % SS) * SD; };
    auto bar = [&](long long p) { return bars + (p - pbase) % SS; };
    auto parity = [&](long long p) { return (unsigned)(((p - pbase) / SS) & 1); };
    auto issue = [&](long long p) {  // one thread
        if (p < 0 || p >= QN) {  // outside the box: the stage arrives without a copy
            mbar_expect_tx(bar(p), 0u);
            return;
        }
        const bool own = ACCUM && p >= q0 && p < q1;
        double *st = stage(p);
        mbar_expect_tx(bar(p), (unsigned)(8 * ((xhi - xlo) + (own ? ylen : 0))));
        tma_load(st + (xlo - p0 + GD), x + p * LEN + xlo, (unsigned)(8 * (xhi - xlo)), bar(p));
        if (own) tma_load(st + PITCH, y + p * LEN + p0, (unsigned)(8 * ylen), bar(p));
    };
    long long issued = pbase - 1;
    if (tid == 0) {
        const long long stop = min(plast, pbase + SS - 1);
        for (long long p = pbase; p <= stop; ++p) issue(p);
        issued = stop;
    }

    // inner factors of the thread's positions (registers, fixed for the launch)
    const double *__restrict__ tab = a.tables;
    const double alpha = a.d_alpha ? __ldg(a.d_alpha) : 1.0;
    PosRegs<VS> g;
    int pos[VS], lp[VS];
    bool act[VS];
#pragma unroll
    for (int v = 0; v < VS; ++v) {
        pos[v] = (int)p0 + v * ST + tid;
        act[v] = pos[v] < LEN;
        int xi[KI];
        inner_decode(act[v] ? pos[v] : LEN - 1, xi);
        g.D0[v] = 0.0;
        chunk_prologue<0, TRANS, VS>(a, alpha, tab, xi, v, g);
        lp[v] = v * ST + tid;  // index in the staged tile; an idle position reads, writes nothing
    }

    bool ok = true;
    long long waited = pbase - 1;  // rows whose copies this thread has seen land
    for (long long p = pbase; p < q0 + HB && ok; ++p) {
        ok = mbar_wait_bounded(bar(p), parity(p), CUFSP_KRON_SLAB_WAIT_TRIES);
        if (ok) waited = p;
    }
    for (long long q = q0; q < q1; ++q) {
        if (ok) ok = mbar_wait_bounded(bar(q + HB), parity(q + HB), CUFSP_KRON_SLAB_WAIT_TRIES);
        if (!ok) {
            failed = 1;
        } else {
            waited = q + HB;
            int z[NO];
            outer_decode(q, z);
            double G[NR], Gd[NR];
            row_words<0, TRANS>(tab, z, G, Gd);
            const double *rowp[2 * HB + 1];
#pragma unroll
            for (int k = 0; k <= 2 * HB; ++k) rowp[k] = stage(q - HB + k);
            const double *xs = rowp[HB] + GD;
            const double *ys = rowp[HB] + PITCH;  // y tile: index lp
            double xv[VS], acc[VS], dg[VS];
#pragma unroll
            for (int v = 0; v < VS; ++v) {
                xv[v] = xs[lp[v]];
                acc[v] = 0.0;
                dg[v] = g.D0[v];
            }
            slab_terms<0, TRANS>(rowp, g, G, lp, xv, acc);
            rows_diag<0, VS>(g, Gd, dg);
#pragma unroll
            for (int v = 0; v < VS; ++v) {
                if (act[v]) {
                    double r = fma(-dg[v], xv[v], acc[v]);
                    if (ACCUM) r += ys[lp[v]];
                    __stcs(y + q * LEN + pos[v], r);
                }
            }
        }
        __syncthreads();  // the stage of row q - HB is consumed
        if (failed) break;
        if (tid == 0 && issued < plast) {
            ++issued;
            fence_proxy_async();
            issue(issued);
        }
    }
    if (tid == 0) {
        // every issued copy must land before the CTA's shared memory is released
        bool bad = failed != 0;
        for (long long p = waited + 1; p <= issued; ++p)
            if (!mbar_wait_bounded(bar(p), parity(p), 1 << 20)) bad = true;
        if (bad && a.err) atomicExch(a.err, 1);
    }
}

}  // namespace cufsp_kron

extern "C" __global__ void __launch_bounds__(CUFSP_KRON_SLAB_T, CUFSP_KRON_SLAB_MINB) cufsp_kron_slab_accum(
    const CufspKronRtcArgs a, const double *__restrict__ x, double *__restrict__ y) {
    cufsp_kron::kron_slab<true, false>(a, x, y);
}

extern "C" __global__ void __launch_bounds__(CUFSP_KRON_SLAB_T, CUFSP_KRON_SLAB_MINB) cufsp_kron_slab_set(
    const CufspKronRtcArgs a, const double *__restrict__ x, double *__restrict__ y) {
    cufsp_kron::kron_slab<false, false>(a, x, y);
}

extern "C" __global__ void __launch_bounds__(CUFSP_KRON_SLAB_T, CUFSP_KRON_SLAB_MINB) cufsp_kron_slabT_set(
    const CufspKronRtcArgs a, const double *__restrict__ x, double *__restrict__ y) {
    cufsp_kron::kron_slab<false, true>(a, x, y);
}
#endif  // CUFSP_KRON_SLAB

#endif  // __CUDACC_RTC__
#endif  // CUFSP_KRON_RTC_CUH
