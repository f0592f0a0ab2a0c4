// cufsp_kron.cu -- matrix-free generator action for factorised propensities (KRONECKER format).
//
// Replaces SDKronMatSet::action / fspmat_sdkron_mv (src/fspmat_kron_kernels.cu:31-129):
//   y[i] (+)= alpha * sum_r c_r ( x[i - d_r] * prod_s f_{r,s}(x_s - nu_{r,s}) * 1{x - nu_r in box}
//                                - x[i]       * prod_s f_{r,s}(x_s) )
// with d_r = sum_s nu_{r,s} * stride_s.
//
// Design (B200, FP64, HBM-bound; the only DRAM traffic is x once and y once or twice):
//  * The state index is split as i = q * L + p.  p (the "inner" position) covers the first k
//    species, q (the "row") the rest.  Each warp owns a fixed chunk of 32*V consecutive inner
//    positions for the whole launch and sweeps rows q = q0, q0 + S, ...; the inner factor products
//    prod_{s<k} f_{r,s} of its V positions per lane are computed once, into registers.
//  * The row-uniform outer products G_r(q) = prod_{s>=k} f_{r,s} (and the shifted ones, zero when
//    the outer part of x - nu_r leaves the box) are tabulated at create time (Q x NR doubles2, L2
//    resident).  Per row, lane r reads G_r(q) once, multiplies by c_r, and publishes it through a
//    per-warp shared-memory slot: no integer division or table walk per state or per row.
//  * Per state and reaction the work is one gather x[i - d_r] and three FP64 operations; reaction
//    counts are template parameters so no padded reaction costs anything.
//  * All warps sweep the rows in one global order (row stride S = warps / chunks), so the planes
//    addressed by the shifted gathers were brought into L2 by a neighbouring warp moments earlier.
//    x is read through the read-only path, y with evict-first hints.
//  * Gather indices are clamped into [0, n); a neighbour outside the box has a zero coefficient
//    (zero inner factor or zero outer table entry), so all loads of a row issue up front.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include <sstream>

#include "cufsp_internal.h"
#define CUFSP_KRON_RTC_MAX_R 64
#include "cufsp_kron_rtc.cuh"
#include "cufsp_march.h"

namespace cufsp {

constexpr int kKronThreads = 128;
constexpr int kKronWarps = kKronThreads / 32;

struct KronArgs {
    const double *__restrict__ tables;  // [nr][tab_stride]
    const int *__restrict__ nu;         // [nr][ns]
    const double2 *__restrict__ gtab;   // [Q][NR] (shifted, unshifted) outer factor products
    const double *__restrict__ d_alpha; // nullable device scalar multiplying alpha
    const int *__restrict__ d_skip;     // nullable: return at once when *d_skip != 0
    int n;
    int tab_stride;
    int ns, nr, k;
    int L, n_chunks;
    int q_begin, q_end;
    int q_safe_lo, q_safe_hi;  // rows whose gathers i - d_r all lie inside [0, n): no clamping
    int pf_dist;               // L2 prefetch distance in row iterations (0: off)
    int dims[CUFSP_MAX_SPECIES];
    int tab_off[CUFSP_MAX_SPECIES];
    int delta[CUFSP_MAX_REACTIONS];
    double coef[CUFSP_MAX_REACTIONS];
    int gid[CUFSP_MAX_REACTIONS];  // diagonal group of each reaction (same inner factor table)
    int rep[CUFSP_MAX_REACTIONS];  // first reaction of each group
};

// Asynchronous bulk prefetch of [p, p + bytes) into L2 by the TMA unit (16-byte granules).
__device__ __forceinline__ void prefetch_l2_bulk(const void *p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Prefetch this warp's chunk of row q of `v` (n doubles) into L2.  The bulk prefetch needs a
// 16-byte aligned address and size, and v itself may be only 8-byte aligned (a Krylov basis
// vector at an odd offset), so the byte range is shrunk to 16-byte boundaries inside [v, v + n).
template <int V>
__device__ __forceinline__ void prefetch_row_chunk(const double *v, int n, int q, int L, int p_chunk) {
    const long long b = (long long)q * L + p_chunk;
    long long e = b + 32 * V;
    const long long row_end = (long long)(q + 1) * L;
    if (e > row_end) e = row_end;
    const unsigned long long base = reinterpret_cast<unsigned long long>(v);
    const unsigned long long lo_lim = (base + 15ull) & ~15ull, hi_lim = (base + 8ull * (unsigned long long)n) & ~15ull;
    unsigned long long lo = (base + 8ull * (unsigned long long)b) & ~15ull;
    unsigned long long hi = (base + 8ull * (unsigned long long)e + 15ull) & ~15ull;
    if (lo < lo_lim) lo = lo_lim;
    if (hi > hi_lim) hi = hi_lim;
    if (hi > lo) prefetch_l2_bulk(reinterpret_cast<const void *>(lo), (unsigned)(hi - lo));
}

// Loads of one row for one lane: x and y at i0 .. i0 + V - 1 and the gathers x[i0 + v - d_r]
// (clamped into [0, n) unless SAFE, i.e. unless the row is known to keep them in range).
template <int NR, int V, bool ACCUM, bool SAFE>
__device__ __forceinline__ void kron_load_row(const KronArgs &a, const double *__restrict__ x,
                                              const double *__restrict__ y, int i0, int nm1, double (&xv)[V],
                                              double (&yv)[V], double (&xg)[NR][V]) {
    if (V >= 2) {
#pragma unroll
        for (int v = 0; v < V; v += 2) {
            const double2 t = __ldg(reinterpret_cast<const double2 *>(x + i0 + v));
            xv[v] = t.x;
            xv[(v + 1) % V] = t.y;
            if (ACCUM) {
                const double2 u = __ldcs(reinterpret_cast<const double2 *>(y + i0 + v));
                yv[v] = u.x;
                yv[(v + 1) % V] = u.y;
            }
        }
    } else {
        xv[0] = __ldg(x + i0);
        if (ACCUM) yv[0] = __ldcs(y + i0);
    }
    const double *xb = x + i0;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const int d = a.delta[r];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            if (SAFE) {
                xg[r][v] = __ldg(xb + (v - d));
            } else {
                const int src = min(max(i0 + v - d, 0), nm1);
                xg[r][v] = __ldg(x + src);
            }
        }
    }
}

// y[i0 + v] (+)= sum_r wa_r Fa_r x[i - d_r] - x[i] sum_g wb_g Fb_g for one row, where the
// diagonal runs over groups g of reactions sharing one inner factor table.
template <int NR, int NG, int V, bool ACCUM>
__device__ __forceinline__ void kron_row_out(const double *wa, const double *wb, const double (&Fa)[V][NR],
                                             const double (&Fb)[V][NG], const double (&xv)[V],
                                             const double (&yv)[V], const double (&xg)[NR][V], double *yo) {
    double acc[V], dg[V];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = dg[v] = 0.0;
#pragma unroll
    for (int g = 0; g < NG; ++g) {
        const double w = wb[g];
#pragma unroll
        for (int v = 0; v < V; ++v) dg[v] = fma(w, Fb[v][g], dg[v]);
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const double w = wa[r];
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = fma(w * Fa[v][r], xg[r][v], acc[v]);
    }
    double out[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        out[v] = fma(-dg[v], xv[v], acc[v]);
        if (ACCUM) out[v] += yv[v];
    }
    if (V >= 2) {
#pragma unroll
        for (int v = 0; v < V; v += 2)
            __stcs(reinterpret_cast<double2 *>(yo + v), make_double2(out[v], out[(v + 1) % V]));
    } else {
        __stcs(yo, out[0]);
    }
}

#ifndef CUFSP_KRON_MINB
#define CUFSP_KRON_MINB 1
#endif
// Per-warp shared words per row: wa[NR] (shifted), wt[NR] (unshifted, per reaction), wb[NG] (grouped).
template <int NR, int NG>
struct KronRowWords {
    static constexpr int kStride = 2 * NR + NG;
};

template <int NR, int NG, int V, bool ACCUM>
__global__ void __launch_bounds__(kKronThreads, CUFSP_KRON_MINB) k_kron_mv(const KronArgs a, const double *__restrict__ x,
                                                                          double *__restrict__ y) {
    constexpr int RS = KronRowWords<NR, NG>::kStride;
    __shared__ double wsm[kKronWarps][2 * RS];
    if (a.d_skip && *a.d_skip) return;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gwarp = blockIdx.x * kKronWarps + wib;
    const int nwarps = gridDim.x * kKronWarps;
    const int rstride = nwarps / a.n_chunks;
    const int chunk = gwarp % a.n_chunks;
    const int rowoff = gwarp / a.n_chunks;
    if (rowoff >= rstride) return;  // whole warp leaves; no CTA-wide barrier follows

    const int p0 = chunk * (32 * V) + lane * V;
    const bool active = p0 < a.L;  // L is a multiple of V, so p0 + V - 1 < L as well

    // Inner factor products of this lane's V positions, fixed for the whole launch: shifted ones per
    // reaction (Fa) and unshifted ones per diagonal group (Fb, from the group's first reaction).
    double Fa[V][NR], Fb[V][NG];
#pragma unroll
    for (int v = 0; v < V; ++v) {
#pragma unroll
        for (int r = 0; r < NR; ++r) Fa[v][r] = 1.0;
#pragma unroll
        for (int g = 0; g < NG; ++g) Fb[v][g] = 1.0;
        int rem = min(p0 + v, a.L - 1);
        for (int s = 0; s < a.k; ++s) {
            const int d = a.dims[s];
            const int xs = rem % d;
            rem /= d;
            const double *t = a.tables + a.tab_off[s];
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const double *tr = t + r * a.tab_stride;
                const int xsh = xs - __ldg(a.nu + r * a.ns + s);
                Fa[v][r] = (xsh < 0 || xsh >= d) ? 0.0 : Fa[v][r] * __ldg(tr + xsh);
            }
#pragma unroll
            for (int g = 0; g < NG; ++g) Fb[v][g] *= __ldg(t + a.rep[g] * a.tab_stride + xs);
        }
    }

    const double cl = (lane < NR) ? a.coef[lane] * (a.d_alpha ? __ldg(a.d_alpha) : 1.0) : 0.0;
    const int my_gid = (lane < NR) ? a.gid[lane] : -1;
    const int nm1 = a.n - 1;
    double *myw = wsm[wib];
    // The grid sweeps the rows in one global order with stride rstride.
    int q = a.q_begin + rowoff;
    const int q_stop = a.q_end, qstep = rstride;
    const int p_chunk = chunk * (32 * V);
    if (lane == 0) {  // start the L2 prefetch pipeline: the first pf_dist rows of this warp
        for (int d = 0; d < a.pf_dist; ++d) {
            const int qq = q + d * qstep;
            if (qq >= q_stop) break;
            prefetch_row_chunk<V>(x, a.n, qq, a.L, p_chunk);
            if (ACCUM) prefetch_row_chunk<V>(y, a.n, qq, a.L, p_chunk);
        }
    }
    // Two rows per iteration (q and q + qstep): twice the independent loads in flight per warp.
    double2 gA = make_double2(0.0, 0.0), gB = gA;
    if (lane < NR && q < q_stop) gA = __ldg(a.gtab + (size_t)q * NR + lane);
    if (lane < NR && q + qstep < q_stop) gB = __ldg(a.gtab + (size_t)(q + qstep) * NR + lane);
    for (; q < q_stop; q += 2 * qstep) {
        const int q2 = q + qstep;
        const bool has2 = q2 < q_stop;
        const double2 g0 = gA, g1 = gB;
        if (lane < NR && q + 2 * qstep < q_stop) gA = __ldg(a.gtab + (size_t)(q + 2 * qstep) * NR + lane);
        if (lane < NR && q + 3 * qstep < q_stop) gB = __ldg(a.gtab + (size_t)(q + 3 * qstep) * NR + lane);
        if (lane == 0 && a.pf_dist > 0) {
            for (int d = 0; d < 2; ++d) {
                const int qq = q + (a.pf_dist + d) * qstep;
                if (qq < q_stop) {
                    prefetch_row_chunk<V>(x, a.n, qq, a.L, p_chunk);
                    if (ACCUM) prefetch_row_chunk<V>(y, a.n, qq, a.L, p_chunk);
                }
            }
        }
        const int i0 = q * a.L + p0, i1 = q2 * a.L + p0;
        // warp-uniform: both rows' gathers stay inside [0, n) -> no clamping code
        const bool safe = q >= a.q_safe_lo && (has2 ? q2 : q) < a.q_safe_hi;
        double xv0[V], yv0[V], xg0[NR][V], xv1[V], yv1[V], xg1[NR][V];
        if (active) {
            if (safe) {
                kron_load_row<NR, V, ACCUM, true>(a, x, y, i0, nm1, xv0, yv0, xg0);
                if (has2) kron_load_row<NR, V, ACCUM, true>(a, x, y, i1, nm1, xv1, yv1, xg1);
            } else {
                kron_load_row<NR, V, ACCUM, false>(a, x, y, i0, nm1, xv0, yv0, xg0);
                if (has2) kron_load_row<NR, V, ACCUM, false>(a, x, y, i1, nm1, xv1, yv1, xg1);
            }
        }
        // row words: wa_r = c_r Ga_r(q); wb_g = sum over the group's reactions of c_r Gb_r(q)
        if (lane < NR) {
            myw[lane] = cl * g0.x;
            myw[RS + lane] = cl * g1.x;
            if (NG == NR) {
                myw[2 * NR + lane] = cl * g0.y;
                myw[RS + 2 * NR + lane] = cl * g1.y;
            } else {
                myw[NR + lane] = cl * g0.y;
                myw[RS + NR + lane] = cl * g1.y;
            }
        }
        if (NG != NR) {
            __syncwarp();
            if (lane < NG) {
                double s0 = 0.0, s1 = 0.0;
                for (int r = 0; r < NR; ++r) {
                    const bool mine = a.gid[r] == lane;
                    s0 += mine ? myw[NR + r] : 0.0;
                    s1 += mine ? myw[RS + NR + r] : 0.0;
                }
                myw[2 * NR + lane] = s0;
                myw[RS + 2 * NR + lane] = s1;
            }
        }
        (void)my_gid;
        __syncwarp();
        if (active) {
            kron_row_out<NR, NG, V, ACCUM>(myw, myw + 2 * NR, Fa, Fb, xv0, yv0, xg0, y + i0);
            if (has2) kron_row_out<NR, NG, V, ACCUM>(myw + RS, myw + RS + 2 * NR, Fa, Fb, xv1, yv1, xg1, y + i1);
        }
        __syncwarp();
    }
}

struct KronData {
    int64_t n = 0;
    int ns = 0, nr = 0, k = 0, L = 0, Q = 0, V = 1, NR = 1, n_chunks = 1;
    int tab_stride = 0;
    double *d_tables = nullptr;
    int *d_nu = nullptr;
    double2 *d_gtab = nullptr;
    std::vector<int> dims, tab_off, delta;
    int64_t halo = 0;
    int grid_full = 0;
    int q_safe_lo = 0, q_safe_hi = 0;
    int pf_dist = 4;
    int NG = 1;                         // diagonal groups as compiled (2, 4 or NR)
    std::vector<int> gid, rep;          // per reaction / per group
    // TMA-fed marching fast path (cufsp_kron_march.cu)
    bool march = false;
    MarchArgs ma;       // constant part of the launch arguments
    int march_V = 1, march_threads = 0, march_grid = 0;
    size_t march_smem = 0;
    int *h_err = nullptr, *d_err = nullptr;  // watchdog word of the march kernel (mapped host memory)
    double2 *d_gtab_march = nullptr;  // only when the marching split differs from k
    // runtime-specialised plane kernel (cufsp_kron_plane.cu), when the network has its shape
    PlaneData *plane = nullptr;
    std::string plane_why;
    // kernel specialised for the network and box (cufsp_kron_rtc.cuh), for the other networks
    std::shared_ptr<RtcModule> rtc;
    double *d_rtc_tab = nullptr;  // packed tabulated factors
    int rtc_grid = 0;
    std::string rtc_why;
    bool rtc_tried = false;       // built at the first transposed action (or at create when it serves the forward)
    bool rtc_forward = false;     // CUFSP_KRON_RTC=1: it also serves the forward action
    // row kernels of the same module (cufsp_kron_rows_*): inner factors fixed per lane
    bool rows_forward = false;    // they serve the forward action
    bool rows_transpose = false;  // and the transposed one
    int rows_k = 1;               // inner species
    int64_t rows_L = 1;           // inner positions per row
    int rows_grid = 0;
    // slab kernels of the same module (cufsp_kron_slab_*): the row kernels' arithmetic on TMA-staged rows
    int slab_grid = 0, slab_threads = 0;
    size_t slab_smem = 0;
    const ModelHost *model = nullptr;  // the generator's model (outlives this object), for the lazy build
};

// Outer factor table for the inner split k: G[q][r] = (prod_{s>=k} f_{r,s}(x_s - nu_{r,s}), or 0
// when that leaves the box; prod_{s>=k} f_{r,s}(x_s)) for every row q of n / prod_{s<k} n_s.
static std::vector<double2> outer_table(const ModelHost &m, const KronData *kd, int k) {
    int64_t L = 1;
    for (int s = 0; s < k; ++s) L *= kd->dims[s];
    const int64_t Q = m.n / L;
    std::vector<double2> g((size_t)Q * kd->NR, make_double2(0.0, 0.0));
    std::vector<int> xs(m.ns, 0);
    for (int64_t q = 0; q < Q; ++q) {
        int64_t rem = q;
        for (int s = k; s < m.ns; ++s) {
            xs[s] = (int)(rem % kd->dims[s]);
            rem /= kd->dims[s];
        }
        for (int r = 0; r < m.nr; ++r) {
            const double *tr = m.tables.data() + (size_t)r * m.tab_stride;
            double ga = 1.0, gb = 1.0;
            bool ok = true;
            for (int s = k; s < m.ns; ++s) {
                const double *t = tr + m.tab_off[s];
                gb *= t[xs[s]];
                const int xsh = xs[s] - m.nu[(size_t)r * m.ns + s];
                if (xsh < 0 || xsh >= kd->dims[s]) ok = false;
                else ga *= t[xsh];
            }
            g[(size_t)q * kd->NR + r] = make_double2(ok ? ga : 0.0, gb);
        }
    }
    return g;
}

// Plan the marching kernel: the slowest species is the marching axis, rows of L = prod_{s<k} n_s
// inner positions fill W = L / (32 V) warps exactly, plane shifts span at most 2 planes each way.
static void plan_march(const ModelHost &m, KronData *kd) {
    kd->march = false;
    // Opt-in (CUFSP_KRON_MARCH=1): on the 255^3 mass-action workload this kernel still trails the
    // register/L1 kernel (about 200 us vs 147 us), so the latter stays the default.
    const char *ev = getenv("CUFSP_KRON_MARCH");
    if (!ev || atoi(ev) == 0) return;
    const int ns = m.ns;
    if (ns < 2 || kd->NR > 16) return;
    const int zs = ns - 1, Z = kd->dims[zs];
    const int64_t P = m.n / Z;
    int k = -1, V = 0, W = 0;
    int64_t L = 1;
    for (int kk = 1; kk <= zs && k < 0; ++kk) {
        L *= kd->dims[kk - 1];
        for (int vv = 1; vv <= 2 && k < 0; ++vv) {
            if (vv == 2 && kd->NR > 12) continue;
            if (L % (32 * vv) == 0 && L / (32 * vv) <= 8) {
                k = kk;
                V = vv;
                W = (int)(L / (32 * vv));
            }
        }
    }
    if (k < 0 || P % L != 0 || (P % 2) != 0) return;
    const int RP = (int)(P / L);
    std::vector<int> dz(m.nr), drow(m.nr), dp(m.nr);
    int hz_lo = 0, hz_hi = 0, hr_lo = 0, hr_hi = 0, gmax = 0;
    for (int r = 0; r < m.nr; ++r) {
        int64_t p = 0, row = 0, st = 1, rst = 1;
        for (int s = 0; s < k; ++s) {
            p += (int64_t)m.nu[(size_t)r * ns + s] * st;
            st *= kd->dims[s];
        }
        for (int s = k; s < zs; ++s) {
            row += (int64_t)m.nu[(size_t)r * ns + s] * rst;
            rst *= kd->dims[s];
        }
        const int d = m.nu[(size_t)r * ns + zs];
        if (std::llabs(p) >= L || std::llabs(row) >= RP || std::abs(d) > 2) return;  // not a near neighbour
        dz[r] = d;
        drow[r] = (int)row;
        dp[r] = (int)p;
        hz_lo = std::max(hz_lo, d);
        hz_hi = std::max(hz_hi, -d);
        hr_lo = std::max(hr_lo, (int)row);
        hr_hi = std::max(hr_hi, (int)-row);
        gmax = std::max(gmax, (int)std::llabs(p));
    }
    const int slots = hz_lo + hz_hi + 2;
    if (slots > kMarchMaxSlots) return;
    const int guard = std::max(2, (gmax + 1) & ~1);
    const size_t budget = 100 * 1024;
    int R = 0;
    for (int cand : {8, 6, 4, 2, 1}) {  // <= kMarchMaxR; one outer-factor entry per thread
        if (cand > RP || cand > kMarchMaxR || cand * kd->NR > 32 * W) continue;
        const size_t se = 2 * (size_t)guard + (size_t)(cand + hr_lo + hr_hi) * L;
        const size_t bytes = slots * se * 8 + (size_t)cand * kd->NR * 16;
        if (bytes <= budget) {
            R = cand;
            break;
        }
    }
    if (R == 0) return;
    MarchArgs &a = kd->ma;
    std::memset(&a, 0, sizeof(a));
    a.n = (int)m.n;
    a.P = (int)P;
    a.L = (int)L;
    a.RP = RP;
    a.Z = Z;
    a.ns = ns;
    a.k = k;
    a.tab_stride = m.tab_stride;
    a.R = R;
    a.hr_lo = hr_lo;
    a.hr_hi = hr_hi;
    a.hz_lo = hz_lo;
    a.hz_hi = hz_hi;
    a.slots = slots;
    a.guard = guard;
    a.slot_elems = 2 * guard + (R + hr_lo + hr_hi) * (int)L;
    a.row_tiles = (RP + R - 1) / R;
    for (int s = 0; s < CUFSP_MAX_SPECIES; ++s) {
        a.dims[s] = s < ns ? kd->dims[s] : 1;
        a.tab_off[s] = s < ns ? m.tab_off[s] : 0;
    }
    for (int r = 0; r < m.nr; ++r) {
        a.dz[r] = dz[r];
        a.soff[r] = (hr_lo - drow[r]) * (int)L - dp[r];
    }
    kd->march_V = V;
    kd->march_threads = 32 * W;
    kd->march_smem = (size_t)slots * a.slot_elems * 8 + (size_t)R * kd->NR * 16;
    MarchKernel kern[2] = {pick_march_kernel(kd->NR, V, false), pick_march_kernel(kd->NR, V, true)};
    if (!kern[0] || !kern[1]) return;
    int occ = 0;
    for (MarchKernel kf : kern) {
        if (cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kd->march_smem) != cudaSuccess)
            return;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern[1], kd->march_threads, kd->march_smem) != cudaSuccess ||
        occ < 1)
        return;
    const int resident = device_info().sm_count * occ;
    const int zsegs = std::max(1, std::min(Z, resident / a.row_tiles));
    a.zseg = (Z + zsegs - 1) / zsegs;
    kd->march_grid = a.row_tiles * ((Z + a.zseg - 1) / a.zseg);
    if (!(kd->h_err = watch_word_alloc(&kd->d_err))) return;
    kd->march = true;
}

using KronKernel = void (*)(const KronArgs, const double *, double *);

namespace {
const char *kKronRtcSource =
#include "cufsp_kron_rtc_src.inc"
    ;
int env_or(const char *name, int dflt) {
    const char *v = getenv(name);
    return v ? atoi(v) : dflt;
}
}  // namespace

// Compiles the KRONECKER kernel specialised for this network and box (cufsp_kron_rtc.cuh): the kind
// of every factor (ones, identity, table), the packed tables it reads, the shifts and the box as
// constants.  Sets kd->rtc, or the reason in kd->rtc_why.
static void kron_build_rtc(const ModelHost &m, KronData *kd) {
    kd->rtc_tried = true;
    if (env_or("CUFSP_KRON_RTC", -1) == 0) {
        kd->rtc_why = "disabled (CUFSP_KRON_RTC=0)";
        return;
    }
    if (m.nr > CUFSP_KRON_RTC_MAX_R) {
        kd->rtc_why = "more than 64 reactions";
        return;
    }
    const int ns = m.ns, nr = m.nr;
    std::vector<int> kind((size_t)nr * ns, 0), toff((size_t)nr * ns, 0);
    std::vector<double> packed;
    for (int r = 0; r < nr; ++r)
        for (int s = 0; s < ns; ++s) {
            const double *t = m.tables.data() + (size_t)r * m.tab_stride + m.tab_off[s];
            bool ones = true, ident = true;
            for (int x = 0; x <= m.bounds[s]; ++x) {
                if (t[x] != 1.0) ones = false;
                if (t[x] != (double)x) ident = false;
            }
            const size_t k = (size_t)r * ns + s;
            kind[k] = ones ? 0 : (ident ? 1 : 2);
            if (kind[k] == 2) {
                toff[k] = (int)packed.size();
                packed.insert(packed.end(), t, t + m.bounds[s] + 1);
            }
        }
    std::vector<int64_t> stride(ns);
    int64_t st = 1;
    for (int s = 0; s < ns; ++s) {
        stride[s] = st;
        st *= (int64_t)m.bounds[s] + 1;
    }
    const int chunk = std::max(1, std::min(nr, env_or("CUFSP_KRON_RTC_CHUNK", 5)));
    const int minb = std::max(1, std::min(8, env_or("CUFSP_KRON_RTC_MINB", 2)));
    const bool tab_smem = packed.size() * sizeof(double) <= 40960;
    // Row kernels: the inner species are the leading ones up to the last, while a row stays within
    // 65,536 positions.
    int rk = 1;
    int64_t rL = (int64_t)m.bounds[0] + 1;
    while (rk + 1 < ns && rL * ((int64_t)m.bounds[rk] + 1) <= 65536) rL *= (int64_t)m.bounds[rk++] + 1;
    // Terms as the kernel forms them: reactions with one shift whose outer factors are all ones share
    // a gather.  Positions per lane from the per-lane register need (terms x positions): 4 up to 12
    // terms (one 8-warp CTA per SM, 40+ loads in flight per lane: 3.25 TB/s on the 12-reaction gene
    // network at 8.4M states, against 2.88 at 2 positions and 2 CTAs/SM, 2.43 at 1 and 3 CTAs/SM).
    int n_terms = 0;
    {
        std::vector<int64_t> merged;
        for (int r = 0; r < nr; ++r) {
            bool outer_one = true;
            for (int s2 = rk; s2 < ns; ++s2)
                if (m.nu[(size_t)r * ns + s2] != 0 || kind[(size_t)r * ns + s2] != 0) outer_one = false;
            int64_t d = 0;
            for (int s2 = 0; s2 < ns; ++s2) d += (int64_t)m.nu[(size_t)r * ns + s2] * stride[s2];
            if (!outer_one) {
                ++n_terms;
            } else if (std::find(merged.begin(), merged.end(), d) == merged.end()) {
                merged.push_back(d);
                ++n_terms;
            }
        }
    }
    int rv = env_or("CUFSP_KRON_ROWS_V", n_terms <= 12 ? 4 : (n_terms <= 24 ? 2 : 1));
    rv = rv >= 4 ? 4 : (rv == 2 ? 2 : 1);
    while (rv > 1 && 32LL * rv > rL) rv /= 2;  // short rows: no idle lanes
    const int rchunk = std::max(1, std::min(nr, env_or("CUFSP_KRON_ROWS_CHUNK", 12)));
    const int rminb = std::max(1, std::min(8, env_or("CUFSP_KRON_ROWS_MINB", rv == 4 ? 1 : (rv == 2 ? 2 : 3))));
    kd->rows_k = rk;
    kd->rows_L = rL;
    // Slab kernels (rows staged by TMA): rows of at least 64 positions (even: 16-byte copies), cut into
    // tiles of at most 1024 positions (4 per thread); reactions moving the row by at most 2 and the
    // position by at most 512; CTAs = tiles x row segments of at least 8 rows, enough to fill the SMs.
    int slab_h = 0, slab_g = 0;
    const int64_t n_rows = m.n / rL;
    bool slab = env_or("CUFSP_KRON_SLAB", 1) != 0 && ns >= 2 && rL % 2 == 0 && rL >= 64 && n_rows >= 8;
    for (int r = 0; r < nr && slab; ++r) {
        int64_t dp = 0, st2 = 1;
        for (int s2 = 0; s2 < rk; ++s2) {
            dp += (int64_t)m.nu[(size_t)r * ns + s2] * st2;
            st2 *= (int64_t)m.bounds[s2] + 1;
        }
        int64_t dfull = 0;
        for (int s2 = 0; s2 < ns; ++s2) dfull += (int64_t)m.nu[(size_t)r * ns + s2] * stride[s2];
        const int64_t dq = (dfull - dp) / rL;
        if (std::llabs(dq) > 2 || std::llabs(dp) > 512) slab = false;
        slab_h = std::max<int>(slab_h, (int)std::llabs(dq));
        slab_g = std::max<int>(slab_g, (int)std::llabs(dp));
    }
    slab_g = (slab_g + 1) & ~1;
    const int slab_vs = (int)std::max<int64_t>(1, std::min<int64_t>(4, rL / 128));  // >= 4 warps per CTA
    const int slab_t = (int)std::min<int64_t>(256, (rL + 32LL * slab_vs - 1) / (32LL * slab_vs) * 32);
    const int64_t slab_tw = (int64_t)slab_t * slab_vs;
    const int64_t slab_ntile = (rL + slab_tw - 1) / slab_tw;
    int slab_minb = 2;
    const int64_t stage_bytes = 8 * (2 * slab_tw + 2LL * slab_g);
    int slab_s = (int)std::min<int64_t>(8, (110 * 1024) / stage_bytes);
    if (slab_s < 2 * slab_h + 2) {  // one CTA per SM with twice the shared memory
        slab_minb = 1;
        slab_s = (int)std::min<int64_t>(8, (200 * 1024) / stage_bytes);
    }
    slab_s = std::min(slab_s, env_or("CUFSP_KRON_SLAB_S", slab_s));
    if (slab_s < 2 * slab_h + 2) slab = false;
    {
        const int64_t resident = (int64_t)device_info().sm_count * slab_minb;
        const int64_t nseg = std::max<int64_t>(1, std::min<int64_t>(resident / slab_ntile, n_rows / 8));
        if (slab_ntile * nseg < device_info().sm_count) slab = false;  // too few CTAs to fill the GPU
    }
    kd->slab_smem = slab ? (size_t)slab_s * (size_t)stage_bytes : 0;
    kd->slab_threads = slab_t;
    std::ostringstream o;
    o << "#define CUFSP_KRON_MINB " << minb << "\n#define CUFSP_KRON_RTC_MAX_R " << CUFSP_KRON_RTC_MAX_R
      << "\n#define CUFSP_KRON_NS " << ns << "\n#define CUFSP_KRON_NR " << nr << "\n#define CUFSP_KRON_N " << m.n
      << "LL\n#define CUFSP_KRON_CHUNK " << chunk << "\n#define CUFSP_KRON_TS " << std::max<size_t>(1, packed.size())
      << "\n#define CUFSP_KRON_TAB_SMEM " << (tab_smem ? 1 : 0) << "\n#define CUFSP_KRON_K " << rk
      << "\n#define CUFSP_KRON_V " << rv << "\n#define CUFSP_KRON_L " << rL << "LL\n#define CUFSP_KRON_RCHUNK " << rchunk
      << "\n#define CUFSP_KRON_ROWS_MINB " << rminb << "\n#define CUFSP_KRON_SLAB " << (slab ? 1 : 0)
      << "\n#define CUFSP_KRON_SLAB_T " << slab_t << "\n#define CUFSP_KRON_SLAB_VS " << slab_vs
      << "\n#define CUFSP_KRON_SLAB_S " << slab_s << "\n#define CUFSP_KRON_SLAB_H " << slab_h
      << "\n#define CUFSP_KRON_SLAB_G " << slab_g << "\n#define CUFSP_KRON_SLAB_MINB " << slab_minb;
    // Bounded waits of the slab kernels: 2^20 tries unless CUFSP_KRON_SLAB_WAIT_TRIES asks for fewer
    // (the watchdog's own test: 0 makes every wait before a row give up at once).
    if (env_or("CUFSP_KRON_SLAB_SHFL", 1) == 0) o << "\n#define CUFSP_KRON_SLAB_SHFL 0";
    if (const char *ev = getenv("CUFSP_KRON_SLAB_WAIT_TRIES"))
        o << "\n#define CUFSP_KRON_SLAB_WAIT_TRIES " << std::max(0, std::min(1 << 20, atoi(ev)));
    o << "\nnamespace cufsp_kron {\n";
    o << "__device__ __forceinline__ constexpr int ext(int s) {";
    for (int s = 0; s < ns; ++s) o << " if (s == " << s << ") return " << m.bounds[s] + 1 << ";";
    o << " return 1; }\n";
    auto emit2 = [&](const char *name, const std::vector<int> &v) {
        o << "__device__ __forceinline__ constexpr int " << name << "(int r, int s) {";
        for (int r = 0; r < nr; ++r)
            for (int s = 0; s < ns; ++s)
                if (v[(size_t)r * ns + s] != 0)
                    o << " if (r == " << r << " && s == " << s << ") return " << v[(size_t)r * ns + s] << ";";
        o << " return 0; }\n";
    };
    emit2("nu", m.nu);
    emit2("kind", kind);
    emit2("t_off", toff);
    o << "__device__ __forceinline__ constexpr long long shift(int r) {";
    for (int r = 0; r < nr; ++r) {
        int64_t d = 0;
        for (int s = 0; s < ns; ++s) d += (int64_t)m.nu[(size_t)r * ns + s] * stride[s];
        o << " if (r == " << r << ") return " << d << "LL;";
    }
    o << " return 0; }\n}\n";
    std::string why;
    std::vector<std::string> names = {"cufsp_kron_mv_accum",   "cufsp_kron_mv_set",   "cufsp_kron_mvT_set",
                                      "cufsp_kron_rows_accum", "cufsp_kron_rows_set", "cufsp_kron_rowsT_set"};
    if (slab) names.insert(names.end(), {"cufsp_kron_slab_accum", "cufsp_kron_slab_set", "cufsp_kron_slabT_set"});
    auto mod = rtc_module(o.str() + kKronRtcSource, names, why);
    if (!mod) {
        kd->rtc_why = why;
        return;
    }
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void *)mod->kernels[0], 256, 0) != cudaSuccess ||
        occ < 1) {
        cudaGetLastError();
        kd->rtc_why = "specialised kernel does not fit an SM";
        return;
    }
    if (packed.empty()) packed.push_back(0.0);
    if (dev_malloc(&kd->d_rtc_tab, sizeof(double) * packed.size()) != cudaSuccess ||
        cudaMemcpy(kd->d_rtc_tab, packed.data(), sizeof(double) * packed.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        upload_fence() != cudaSuccess) {
        cudaGetLastError();
        kd->rtc_why = "table allocation failed";
        return;
    }
    kd->rtc = mod;
    kd->rtc_grid = device_info().sm_count * occ;
    // Row kernels: a persistent grid whose warp count is a multiple of the chunks per row, so that
    // each warp keeps one chunk (and computes its inner factors once).
    int rocc = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rocc, (const void *)mod->kernels[3], 256, 0) != cudaSuccess ||
        rocc < 1) {
        cudaGetLastError();
        kd->rows_forward = kd->rows_transpose = false;
        return;
    }
    // Slab kernels: every tile of a row in each of as many row segments as CTAs fit (8 rows at least).
    kd->slab_grid = 0;
    if (slab) {
        int socc = 0;
        bool sok = true;
        for (int k = 6; k < 9 && sok; ++k)
            sok = cudaFuncSetAttribute((const void *)mod->kernels[k], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kd->slab_smem) == cudaSuccess;
        if (sok && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&socc, (const void *)mod->kernels[6], slab_t,
                                                                 kd->slab_smem) == cudaSuccess &&
            socc >= 1 && (kd->h_err || (kd->h_err = watch_word_alloc(&kd->d_err)))) {
            const int64_t resident = (int64_t)device_info().sm_count * std::min(socc, 8);
            const int64_t nseg = std::max<int64_t>(1, std::min<int64_t>(resident / slab_ntile, n_rows / 8));
            kd->slab_grid = (int)(slab_ntile * nseg);
        }
        cudaGetLastError();
    }
    const int64_t nch = (rL + 32LL * rv - 1) / (32LL * rv);
    const int64_t resident = (int64_t)device_info().sm_count * rocc;
    const int64_t h = nch / std::gcd<int64_t>(nch, 8);  // CTAs per group of 8h warps = h chunks x 8 rows
    kd->rows_grid = (int)(h <= resident ? (resident / h) * h : resident);
}

template <int NR, int V>
static KronKernel pick_ng(int NG, bool accum) {
    if (NG == 2 && NR > 2) return accum ? k_kron_mv<NR, (NR > 2 ? 2 : NR), V, true> : k_kron_mv<NR, (NR > 2 ? 2 : NR), V, false>;
    if (NG == 4 && NR > 4) return accum ? k_kron_mv<NR, (NR > 4 ? 4 : NR), V, true> : k_kron_mv<NR, (NR > 4 ? 4 : NR), V, false>;
    return accum ? k_kron_mv<NR, NR, V, true> : k_kron_mv<NR, NR, V, false>;
}

#define KRON_CASE(NRv, Vv) \
    case NRv:              \
        return pick_ng<NRv, Vv>(NG, accum);

// NG: diagonal groups as compiled (2, 4 or NR).
static KronKernel pick_kernel(int NR, int NG, int V, bool accum) {
    if (V == 4) {
        switch (NR) {
            KRON_CASE(1, 4) KRON_CASE(2, 4) KRON_CASE(3, 4) KRON_CASE(4, 4) KRON_CASE(5, 4) KRON_CASE(6, 4)
            default: return nullptr;
        }
    }
    if (V == 2) {
        switch (NR) {
            KRON_CASE(1, 2) KRON_CASE(2, 2) KRON_CASE(3, 2) KRON_CASE(4, 2) KRON_CASE(5, 2) KRON_CASE(6, 2)
            KRON_CASE(7, 2) KRON_CASE(8, 2) KRON_CASE(9, 2) KRON_CASE(10, 2) KRON_CASE(11, 2) KRON_CASE(12, 2)
            default: return nullptr;
        }
    }
    switch (NR) {
        KRON_CASE(1, 1) KRON_CASE(2, 1) KRON_CASE(3, 1) KRON_CASE(4, 1) KRON_CASE(5, 1) KRON_CASE(6, 1)
        KRON_CASE(7, 1) KRON_CASE(8, 1) KRON_CASE(9, 1) KRON_CASE(10, 1) KRON_CASE(11, 1) KRON_CASE(12, 1)
        KRON_CASE(13, 1) KRON_CASE(14, 1) KRON_CASE(15, 1) KRON_CASE(16, 1) KRON_CASE(20, 1) KRON_CASE(24, 1)
        KRON_CASE(28, 1) KRON_CASE(32, 1)
        default: return nullptr;
    }
}
#undef KRON_CASE

static int max_v_for(int NR) { return NR <= 6 ? 4 : (NR <= 12 ? 2 : 1); }

cufsp_status kron_create(const ModelHost &m, KronData **out) {
    if (m.nr > CUFSP_MAX_REACTIONS)
        return set_error(CUFSP_ERR_UNSUPPORTED, "KRONECKER format supports at most 32 reactions");
    if (m.n > (int64_t(1) << 30))  // gather indices i - d_r stay inside int32 for n <= 2^30
        return set_error(CUFSP_ERR_UNSUPPORTED, "KRONECKER format supports at most 2^30 states");
    KronData *kd = new KronData();
    kd->n = m.n;
    kd->ns = m.ns;
    kd->nr = m.nr;
    kd->tab_stride = m.tab_stride;
    kd->tab_off = m.tab_off;
    kd->dims.resize(m.ns);
    for (int s = 0; s < m.ns; ++s) kd->dims[s] = m.bounds[s] + 1;
    kd->NR = m.nr <= 16 ? m.nr : (m.nr <= 20 ? 20 : m.nr <= 24 ? 24 : m.nr <= 28 ? 28 : 32);

    // Shifts d_r = sum_s nu_{r,s} * stride_s and the halo max |d_r|.
    std::vector<int64_t> stride(m.ns);
    int64_t st = 1;
    for (int s = 0; s < m.ns; ++s) {
        stride[s] = st;
        st *= kd->dims[s];
    }
    kd->delta.assign(CUFSP_MAX_REACTIONS, 0);
    for (int r = 0; r < m.nr; ++r) {
        int64_t d = 0;
        for (int s = 0; s < m.ns; ++s) d += (int64_t)m.nu[(size_t)r * m.ns + s] * stride[s];
        if (d > m.n || d < -m.n) d = 0;  // such a neighbour is never inside the box (factor 0)
        kd->delta[r] = (int)d;
        kd->halo = std::max<int64_t>(kd->halo, d < 0 ? -d : d);
    }

    // Inner split (k species) and states per lane V: few idle lanes, large V.
    const DeviceInfo &di = device_info();
    int vmax = max_v_for(kd->NR);
    if (const char *ev = getenv("CUFSP_KRON_VMAX")) {  // tuning override: cap states per lane (1, 2, 4)
        const int v = atoi(ev);
        if (v == 1 || v == 2 || v == 4) vmax = std::min(vmax, v);
    }
    double best = 1e300;
    int best_k = 1, best_v = 1;
    int64_t Lk = 1;
    for (int k = 1; k <= m.ns; ++k) {
        Lk *= kd->dims[k - 1];
        if (Lk > 2147483647LL) break;
        for (int V = vmax; V >= 1; V /= 2) {
            if (Lk % V) continue;
            const int64_t w = 32LL * V;
            const int64_t chunks = (Lk + w - 1) / w;
            if (chunks > (int64_t)di.sm_count * 16 && !(k == 1 && V == 1)) continue;
            const double waste = (double)(chunks * w - Lk) / (double)Lk;
            const double score = (1.0 + waste) * (1.0 + 0.5 / V);
            if (score < best - 1e-12) {
                best = score;
                best_k = k;
                best_v = V;
            }
        }
    }
    kd->k = best_k;
    kd->V = best_v;
    int64_t L = 1;
    for (int s = 0; s < best_k; ++s) L *= kd->dims[s];
    kd->L = (int)L;
    kd->Q = (int)(m.n / L);
    kd->n_chunks = (int)((L + 32LL * kd->V - 1) / (32LL * kd->V));
    // Rows q whose gathers stay in [0, n): q L >= max d_r and (q + 1) L <= n + min d_r.
    int64_t dmax = 0, dmin = 0;
    for (int r = 0; r < m.nr; ++r) {
        dmax = std::max<int64_t>(dmax, kd->delta[r]);
        dmin = std::min<int64_t>(dmin, kd->delta[r]);
    }
    kd->q_safe_lo = (int)((dmax + 1 + L - 1) / L);  // +1: odd shifts load the pair one element lower
    kd->q_safe_hi = (int)std::max<int64_t>(0, (m.n + dmin) / L);
    if (const char *ev = getenv("CUFSP_KRON_PF")) {  // tuning override: L2 prefetch distance in rows
        const int v = atoi(ev);
        if (v >= 0 && v <= 64) kd->pf_dist = v;
    }

    const std::vector<double2> g = outer_table(m, kd, best_k);

    // Diagonal groups: reactions whose inner factor tables (species < k) are identical share one
    // per-lane factor, so the diagonal costs one FMA per group and state instead of per reaction.
    kd->gid.assign(CUFSP_MAX_REACTIONS, 0);
    kd->rep.assign(CUFSP_MAX_REACTIONS, 0);
    int ng = 0;
    for (int r = 0; r < m.nr; ++r) {
        int found = -1;
        for (int gg = 0; gg < ng && found < 0; ++gg) {
            const int r2 = kd->rep[gg];
            bool same = true;
            for (int s = 0; s < best_k && same; ++s) {
                const double *a1 = m.tables.data() + (size_t)r * m.tab_stride + m.tab_off[s];
                const double *a2 = m.tables.data() + (size_t)r2 * m.tab_stride + m.tab_off[s];
                same = std::equal(a1, a1 + kd->dims[s], a2);
            }
            if (same) found = gg;
        }
        if (found < 0) {
            found = ng;
            kd->rep[ng++] = r;
        }
        kd->gid[r] = found;
    }
    kd->NG = (ng <= 2 && kd->NR > 2) ? 2 : (ng <= 4 && kd->NR > 4) ? 4 : kd->NR;
    if (kd->NG == kd->NR) {  // no grouping: the diagonal keeps one term per reaction
        for (int r = 0; r < CUFSP_MAX_REACTIONS; ++r) kd->gid[r] = kd->rep[r] = (r < kd->NR ? r : 0);
    }

    int occ = 0;
    KronKernel kern = pick_kernel(kd->NR, kd->NG, kd->V, true);
    if (!kern) {
        kron_destroy(kd);
        return set_error(CUFSP_ERR_UNSUPPORTED, "no KRONECKER kernel for this reaction count");
    }
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kKronThreads, 0);
    if (e != cudaSuccess || occ < 1) occ = 1;
    kd->grid_full = di.sm_count * occ;

    // Tables padded to NR reactions (padding rows are zero: no contribution, in-bounds reads).
    std::vector<double> tabp((size_t)kd->NR * m.tab_stride, 0.0);
    std::copy(m.tables.begin(), m.tables.end(), tabp.begin());
    std::vector<int> nup((size_t)kd->NR * m.ns, 0);
    std::copy(m.nu.begin(), m.nu.end(), nup.begin());
    e = dev_malloc(&kd->d_tables, sizeof(double) * tabp.size());
    if (e == cudaSuccess) e = dev_malloc(&kd->d_nu, sizeof(int) * nup.size());
    if (e == cudaSuccess) e = dev_malloc(&kd->d_gtab, sizeof(double2) * g.size());
    if (e == cudaSuccess) e = cudaMemcpy(kd->d_tables, tabp.data(), sizeof(double) * tabp.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(kd->d_nu, nup.data(), sizeof(int) * nup.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(kd->d_gtab, g.data(), sizeof(double2) * g.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        kron_destroy(kd);
        return cuda_error(e, "kron_create");
    }
    kd->plane = plane_create(m, kd->d_tables, kd->plane_why);
    kd->model = &m;
    // The specialised kernel serves the transposed action (built at its first use).  For the forward
    // action it is opt-in (CUFSP_KRON_RTC=1): it recomputes every propensity from the factors per
    // state, which on the 12-reaction gene network at 8.4M states is issue-bound (1.76 TB/s) where the
    // generic kernel, sharing inner and outer factor products across a row, moves 1.92 TB/s.
    kd->rtc_forward = env_or("CUFSP_KRON_RTC", -1) == 1;
    // Row kernels for the networks the plane kernel does not take (CUFSP_KRON_ROWS=0: off, 1: also
    // below 65,536 states, where the generic kernel is the default to spare small models a compile).
    const int rows_env = env_or("CUFSP_KRON_ROWS", -1);
    kd->rows_forward = !kd->plane && rows_env != 0 && (rows_env == 1 || m.n >= 65536);
    kd->rows_transpose = rows_env != 0 && (rows_env == 1 || m.n >= 65536);
    if ((kd->rtc_forward || kd->rows_forward) && !kd->plane) kron_build_rtc(m, kd);
    plan_march(m, kd);
    if (kd->march && kd->ma.k != kd->k) {  // the marching split needs its own outer table
        const std::vector<double2> gm = outer_table(m, kd, kd->ma.k);
        e = dev_malloc(&kd->d_gtab_march, sizeof(double2) * gm.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(kd->d_gtab_march, gm.data(), sizeof(double2) * gm.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) kd->march = false;
    }
    cudaGetLastError();  // a declined fast path leaves no sticky error behind
    e = upload_fence();
    if (e != cudaSuccess) {
        kron_destroy(kd);
        return cuda_error(e, "kron_create");
    }
    *out = kd;
    return CUFSP_SUCCESS;
}

void kron_destroy(KronData *k) {
    if (!k) return;
    if (k->d_tables) cudaFree(k->d_tables);
    if (k->d_nu) cudaFree(k->d_nu);
    if (k->d_gtab) cudaFree(k->d_gtab);
    if (k->d_gtab_march) cudaFree(k->d_gtab_march);
    if (k->d_rtc_tab) cudaFree(k->d_rtc_tab);
    watch_word_free(k->h_err);
    plane_destroy(k->plane);
    delete k;
}

int kron_watchdog(KronData *k) {
    if (!k) return 0;
    const int pv = k->plane ? plane_watchdog(k->plane) : 0;
    return watch_word_take(k->h_err) | pv;
}

// The plane kernel reads one plane beyond each end of the range it computes.
int64_t kron_halo(const KronData *k) { return k->plane ? std::max<int64_t>(k->halo, plane_size(k->plane)) : k->halo; }
int64_t kron_row_len(const KronData *k) { return k->plane ? plane_size(k->plane) : k->L; }

namespace {
// The specialised kernel is compiled (NVRTC) and its tables copied at its first use -- never while
// `st` is being captured into a graph, where those calls are not allowed: drivers that capture call
// kron_prepare first, and an apply met during a capture falls back to the generic kernels.
void ensure_rtc(KronData *k, cudaStream_t st) {
    if (k->rtc_tried || !k->model) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    if (cs == cudaStreamCaptureStatusNone) kron_build_rtc(*k->model, k);
}
}  // namespace

cufsp_status kron_prepare(KronData *k, const double *coefs, cudaStream_t st, bool transpose) {
    if (transpose || k->rtc_forward || k->rows_forward) ensure_rtc(k, st);
    return k->plane ? plane_prepare(k->plane, coefs, st) : CUFSP_SUCCESS;
}

std::string kron_describe(const KronData *k) {
    if (k->plane) return plane_description(k->plane);
    if (k->rows_forward && k->rtc && k->slab_grid > 0)
        return "slab kernel specialised for the network and box (NVRTC, sm_100a, TMA ring): " +
               std::to_string(k->rows_k) + " inner species, rows of " + std::to_string(k->rows_L) + " positions, " +
               std::to_string(k->slab_grid) + " CTAs x " + std::to_string(k->slab_threads) + " threads, " +
               std::to_string(k->slab_smem) + " B smem; plane kernel not used: " + k->plane_why;
    if (k->rows_forward && k->rtc && k->rows_grid > 0)
        return "row kernel specialised for the network and box (NVRTC, sm_100a): " + std::to_string(k->rows_k) +
               " inner species, rows of " + std::to_string(k->rows_L) + " positions, " + std::to_string(k->rows_grid) +
               " CTAs x 256 threads; plane kernel not used: " + k->plane_why;
    if (k->rtc_forward && k->rtc)
        return "kernel specialised for the network and box (NVRTC, sm_100a), " + std::to_string(k->rtc_grid) +
               " CTAs x 256 threads; plane kernel not used: " + k->plane_why;
    return "k_kron_mv (NR=" + std::to_string(k->NR) + " NG=" + std::to_string(k->NG) + " V=" + std::to_string(k->V) +
           " inner species=" + std::to_string(k->k) + "); plane kernel not used: " + k->plane_why +
           (k->rtc_forward ? "; specialised kernel not used: " + k->rtc_why : std::string());
}

// ---- transposed action (adjoint solves) ---------------------------------------------------------
// (A^T l)(x) = sum_r c_r a_r(x) (l[x + nu_r] 1{x + nu_r in box} - l[x]): the column of the generator
// at state x (outflow a_r(x) to x + nu_r, or out of the box) read as a row.  One thread per state,
// factors from the tables; used by the adjoint gradient, not on the forward hot path.
struct KronTArgs {
    const double *__restrict__ tables;
    const int *__restrict__ nu;  // [NR][ns]
    const double *__restrict__ d_alpha;
    const int *__restrict__ d_skip;
    int n, ns, nr, tab_stride;
    int dims[CUFSP_MAX_SPECIES];
    int tab_off[CUFSP_MAX_SPECIES];
    FastDiv div[CUFSP_MAX_SPECIES];
    int delta[CUFSP_MAX_REACTIONS];
    double coef[CUFSP_MAX_REACTIONS];
};

__global__ void __launch_bounds__(256) k_kron_mvT(const KronTArgs a, const double *__restrict__ x, double *__restrict__ y) {
    if (a.d_skip && *a.d_skip) return;
    const double alpha = a.d_alpha ? __ldg(a.d_alpha) : 1.0;
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
        const double xi = __ldg(x + i);
        double acc = 0.0;
        for (int r = 0; r < a.nr; ++r) {
            double f = a.coef[r];
            bool ok = true;
            const double *tr = a.tables + (size_t)r * a.tab_stride;
            for (int s = 0; s < a.ns; ++s) {
                f *= __ldg(tr + a.tab_off[s] + xs[s]);
                const int t = xs[s] + __ldg(a.nu + r * a.ns + s);
                ok = ok && t >= 0 && t < a.dims[s];
            }
            const double tgt = ok ? __ldg(x + i + a.delta[r]) : 0.0;
            acc = fma(f, tgt - xi, acc);
        }
        y[i] = alpha * acc;
    }
}

// One launch of a row kernel (module kernel index `which`: 3 accumulate, 4 overwrite, 5 transposed) over
// all rows.  Plain 8-byte loads and stores: no alignment requirement on x and y.
static cufsp_status rows_launch(KronData *kd, const double *coefs, double alpha, const double *d_alpha,
                                const int *d_skip, const double *x, double *y, int which, cudaStream_t st) {
    CufspKronRtcArgs r;
    std::memset(&r, 0, sizeof(r));
    r.tables = kd->d_rtc_tab;
    r.d_alpha = d_alpha;
    r.d_skip = d_skip;
    r.q_begin = 0;
    r.q_end = kd->n / kd->rows_L;
    for (int k = 0; k < kd->nr; ++k) r.coef[k] = alpha * coefs[k];
    void *args[] = {&r, (void *)&x, (void *)&y};
    // The slab kernel copies whole rows with 16-byte bulk copies: x and y must be 16-byte aligned.
    if (kd->slab_grid > 0 && ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % 16) == 0) {
        r.err = kd->d_err;
        CUFSP_CUDA_TRY(cudaLaunchKernel((const void *)kd->rtc->kernels[which + 3], dim3(kd->slab_grid),
                                        dim3(kd->slab_threads), args, kd->slab_smem, st));
        return CUFSP_SUCCESS;
    }
    CUFSP_CUDA_TRY(cudaLaunchKernel((const void *)kd->rtc->kernels[which], dim3(kd->rows_grid), dim3(256), args, 0, st));
    return CUFSP_SUCCESS;
}

cufsp_status kron_apply_transpose(KronData *kd, const double *coefs, double alpha, const double *d_alpha,
                                  const int *d_skip, const double *x, double *y, cudaStream_t st) {
    ensure_rtc(kd, st);
    if (kd->rows_transpose && kd->rtc && kd->rows_grid > 0)
        return rows_launch(kd, coefs, alpha, d_alpha, d_skip, x, y, 5, st);
    if (kd->rtc && ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % 16) == 0) {
        CufspKronRtcArgs r;
        std::memset(&r, 0, sizeof(r));
        r.tables = kd->d_rtc_tab;
        r.d_alpha = d_alpha;
        r.d_skip = d_skip;
        r.i_begin = 0;
        r.i_end = kd->n;
        for (int k = 0; k < kd->nr; ++k) r.coef[k] = alpha * coefs[k];
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(kd->rtc_grid, (kd->n / 2 + 256) / 256));
        void *args[] = {&r, (void *)&x, (void *)&y};
        CUFSP_CUDA_TRY(cudaLaunchKernel((const void *)kd->rtc->kernels[2], dim3(grid), dim3(256), args, 0, st));
        return CUFSP_SUCCESS;
    }
    KronTArgs a;
    std::memset(&a, 0, sizeof(a));
    a.tables = kd->d_tables;
    a.nu = kd->d_nu;
    a.d_alpha = d_alpha;
    a.d_skip = d_skip;
    a.n = (int)kd->n;
    a.ns = kd->ns;
    a.nr = kd->nr;
    a.tab_stride = kd->tab_stride;
    for (int s = 0; s < kd->ns; ++s) {
        a.dims[s] = kd->dims[s];
        a.tab_off[s] = kd->tab_off[s];
        a.div[s] = make_fastdiv((uint32_t)kd->dims[s]);
    }
    for (int r = 0; r < kd->nr; ++r) {
        a.delta[r] = kd->delta[r];
        a.coef[r] = alpha * coefs[r];
    }
    const int grid = (int)std::min<int64_t>((kd->n + 255) / 256, (int64_t)device_info().sm_count * 16);
    k_kron_mvT<<<std::max(grid, 1), 256, 0, st>>>(a, x, y);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

cufsp_status kron_apply(KronData *kd, const double *coefs, double alpha, const double *d_alpha, const int *d_skip,
                        const double *x, bool accumulate, double *y, cudaStream_t st, int64_t i_begin, int64_t i_end) {
    if (kd->plane) {
        cufsp_status ps = CUFSP_SUCCESS;
        if (plane_launch(kd->plane, coefs, alpha, d_alpha, d_skip, x, accumulate, y, st, i_begin, i_end, &ps)) return ps;
    }
    const bool full = i_begin == 0 && (i_end < 0 || i_end == kd->n);
    if (kd->march && full && (reinterpret_cast<uintptr_t>(x) % 16) == 0) {
        MarchArgs ma = kd->ma;
        ma.gtab = kd->d_gtab_march ? kd->d_gtab_march : kd->d_gtab;
        ma.tables = kd->d_tables;
        ma.nu = kd->d_nu;
        ma.d_alpha = d_alpha;
        ma.d_skip = d_skip;
        ma.err = kd->d_err;
        for (int r = 0; r < CUFSP_MAX_REACTIONS; ++r) ma.coef[r] = r < kd->nr ? alpha * coefs[r] : 0.0;
        MarchKernel mk = pick_march_kernel(kd->NR, kd->march_V, accumulate);
        if (mk) {
            mk<<<(unsigned)kd->march_grid, (unsigned)kd->march_threads, kd->march_smem, st>>>(ma, x, y);
            CUFSP_CUDA_TRY(cudaGetLastError());
            return CUFSP_SUCCESS;
        }
    }
    if (kd->rows_forward && full) {
        ensure_rtc(kd, st);
        if (kd->rtc && kd->rows_grid > 0) return rows_launch(kd, coefs, alpha, d_alpha, d_skip, x, y, accumulate ? 3 : 4, st);
    }
    if (kd->rtc_forward) ensure_rtc(kd, st);
    if (kd->rtc_forward && kd->rtc &&
        ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % 16) == 0) {
        if (i_end < 0) i_end = kd->n;
        if (i_end <= i_begin) return CUFSP_SUCCESS;
        CufspKronRtcArgs r;
        std::memset(&r, 0, sizeof(r));
        r.tables = kd->d_rtc_tab;
        r.d_alpha = d_alpha;
        r.d_skip = d_skip;
        r.i_begin = i_begin;
        r.i_end = i_end;
        for (int k = 0; k < kd->nr; ++k) r.coef[k] = alpha * coefs[k];
        const int64_t pairs = (i_end - (i_begin & ~(int64_t)1) + 1) / 2;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(kd->rtc_grid, (pairs + 255) / 256));
        void *args[] = {&r, (void *)&x, (void *)&y};
        CUFSP_CUDA_TRY(cudaLaunchKernel((const void *)kd->rtc->kernels[accumulate ? 0 : 1], dim3(grid), dim3(256), args,
                                        0, st));
        return CUFSP_SUCCESS;
    }
    KronArgs a;
    a.tables = kd->d_tables;
    a.nu = kd->d_nu;
    a.gtab = kd->d_gtab;
    a.d_alpha = d_alpha;
    a.d_skip = d_skip;
    a.n = (int)kd->n;
    a.tab_stride = kd->tab_stride;
    a.ns = kd->ns;
    a.nr = kd->nr;
    a.k = kd->k;
    a.L = kd->L;
    // V >= 2 moves x and y in 16-byte pairs; vectors only 8-byte aligned take the V = 1 kernel.
    const bool aligned16 = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % 16) == 0;
    const int V = aligned16 ? kd->V : 1;
    const int n_chunks = (int)((kd->L + 32LL * V - 1) / (32LL * V));
    a.n_chunks = n_chunks;
    if (i_end < 0) i_end = kd->n;
    a.q_begin = (int)(i_begin / kd->L);
    a.q_end = (int)((i_end + kd->L - 1) / kd->L);
    a.q_safe_lo = kd->q_safe_lo;
    a.q_safe_hi = kd->q_safe_hi;
    a.pf_dist = V >= 2 ? kd->pf_dist : 0;  // the bulk L2 prefetch only pays off for paired loads
    for (int s = 0; s < CUFSP_MAX_SPECIES; ++s) {
        a.dims[s] = s < kd->ns ? kd->dims[s] : 1;
        a.tab_off[s] = s < kd->ns ? kd->tab_off[s] : 0;
    }
    for (int r = 0; r < CUFSP_MAX_REACTIONS; ++r) {
        a.delta[r] = r < kd->nr ? kd->delta[r] : 0;
        a.coef[r] = r < kd->nr ? alpha * coefs[r] : 0.0;
        a.gid[r] = kd->gid[r];
        a.rep[r] = kd->rep[r];
    }
    const int rows = a.q_end - a.q_begin;
    if (rows <= 0) return CUFSP_SUCCESS;
    // Enough warps for every chunk, at most the persistent grid, and >= ~4 rows per warp.
    const int64_t min_grid = (n_chunks + kKronWarps - 1) / kKronWarps;
    const int64_t want_warps = (int64_t)n_chunks * ((rows + 3) / 4);
    int64_t grid = (want_warps + kKronWarps - 1) / kKronWarps;
    grid = std::max(grid, min_grid);
    grid = std::min<int64_t>(grid, std::max<int64_t>(kd->grid_full, min_grid));
    KronKernel kern = pick_kernel(kd->NR, kd->NG, V, accumulate);
    if (!kern) return set_error(CUFSP_ERR_UNSUPPORTED, "no KRONECKER kernel for this reaction count");
    kern<<<(unsigned)grid, kKronThreads, 0, st>>>(a, x, y);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

}  // namespace cufsp
