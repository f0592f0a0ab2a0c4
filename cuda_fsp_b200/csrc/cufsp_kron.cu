// cufsp_kron.cu -- matrix-free generator action for factorised propensities (KRONECKER format).
//
// Replaces SDKronMatSet::action / fspmat_sdkron_mv (src/fspmat_kron_kernels.cu:31-129):
//   y[i] (+)= alpha * sum_r c_r ( x[i - d_r] * prod_s f_{r,s}(x_s - nu_{r,s}) * 1{x - nu_r in box}
//                                - x[i]       * prod_s f_{r,s}(x_s) )
// with d_r = sum_s nu_{r,s} * stride_s.
//
// Design (B200, FP64, HBM-bound):
//  * The state index is split as i = q * L + p.  p (the "inner" position) covers the first k
//    species, q (the "row") the rest.  Each warp owns a fixed chunk of 32*V inner positions for
//    the whole launch and sweeps rows q = q0, q0 + S, q0 + 2S, ...: the inner factor products
//    prod_{s<k} f_{r,s} for its V positions per lane are computed ONCE into registers.
//  * Per row, lane r computes the row-uniform outer products prod_{s>=k} f_{r,s} (times c_r)
//    for reaction r and publishes them through a per-warp shared-memory slot, so the per-state
//    work is 3 FP64 ops + 1 gather per reaction; no integer division per state.
//  * All warps of the grid sweep the rows in one global order (row stride S = warps / chunks),
//    so the x planes addressed by the shifted gathers x[i - d_r] were brought into L2 by a
//    neighbouring warp moments earlier: DRAM traffic stays at x once + y once (or twice when
//    accumulating).  x is read through the read-only path, y with evict-first hints.
//  * Gather addresses are clamped into [0, n); a neighbour outside the box has a zero
//    coefficient (factor 0 from the inner or outer validity test), so no predicated loads sit
//    between the address arithmetic and the FMAs and every load of a row is issued up front.
#include <algorithm>
#include <cmath>

#include "cufsp_internal.h"

namespace cufsp {

struct KronArgs {
    const double *__restrict__ tables;  // [nr][tab_stride]
    const int *__restrict__ nu;         // [nr][ns]
    const double *__restrict__ d_alpha; // nullable device scalar multiplying alpha
    const int *__restrict__ d_skip;     // nullable: return at once when *d_skip != 0
    int64_t n;
    int tab_stride;
    int ns, nr, k;
    int L, n_chunks;
    int q_begin, q_end;
    int dims[CUFSP_MAX_SPECIES];
    int tab_off[CUFSP_MAX_SPECIES];
    int delta[CUFSP_MAX_REACTIONS];
    double coef[CUFSP_MAX_REACTIONS];
};

template <int NR, int V, bool ACCUM>
__global__ void __launch_bounds__(256) k_kron_mv(const KronArgs a, const double *__restrict__ x,
                                                 double *__restrict__ y) {
    __shared__ double2 wsm[8][NR];
    if (a.d_skip && *a.d_skip) return;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gwarp = blockIdx.x * 8 + wib;
    const int nwarps = gridDim.x * 8;
    const int rstride = nwarps / a.n_chunks;
    const int chunk = gwarp % a.n_chunks;
    const int rowoff = gwarp / a.n_chunks;
    if (rowoff >= rstride) return;  // whole warp leaves; no CTA-wide barrier follows

    const int p0 = chunk * (32 * V) + lane * V;
    const bool active = p0 < a.L;  // V == 2 only when L is even, so p0 + 1 < L as well

    // Inner factor products for this lane's V positions (fixed for the whole launch).
    double Fa[V][NR], Fb[V][NR];
#pragma unroll
    for (int v = 0; v < V; ++v) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            Fa[v][r] = (r < a.nr) ? 1.0 : 0.0;
            Fb[v][r] = (r < a.nr) ? 1.0 : 0.0;
        }
        int rem = min(p0 + v, a.L - 1);
        for (int s = 0; s < a.k; ++s) {
            const int d = a.dims[s];
            const int xs = rem % d;
            rem /= d;
            const double *t = a.tables + a.tab_off[s];
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                if (r < a.nr) {
                    const double *tr = t + (size_t)r * a.tab_stride;
                    Fb[v][r] *= __ldg(tr + xs);
                    const int xsh = xs - __ldg(a.nu + r * a.ns + s);
                    Fa[v][r] = (xsh < 0 || xsh >= d) ? 0.0 : Fa[v][r] * __ldg(tr + xsh);
                }
            }
        }
    }

    const double alpha_dev = a.d_alpha ? __ldg(a.d_alpha) : 1.0;
    const int64_t nm1 = a.n - 1;
    double2 *myw = wsm[wib];
    for (int q = a.q_begin + rowoff; q < a.q_end; q += rstride) {
        // Row-uniform outer factors, one reaction per lane.
        if (lane < NR) {
            double wa = 0.0, wb = 0.0;
            if (lane < a.nr) {
                double ga = 1.0, gb = 1.0;
                bool ok = true;
                int rem = q;
                const double *tr = a.tables + (size_t)lane * a.tab_stride;
                for (int s = a.k; s < a.ns; ++s) {
                    const int d = a.dims[s];
                    const int xs = rem % d;
                    rem /= d;
                    const double *t = tr + a.tab_off[s];
                    gb *= __ldg(t + xs);
                    const int xsh = xs - __ldg(a.nu + lane * a.ns + s);
                    if (xsh < 0 || xsh >= d) ok = false;
                    else ga *= __ldg(t + xsh);
                }
                const double c = a.coef[lane] * alpha_dev;
                wa = ok ? c * ga : 0.0;
                wb = c * gb;
            }
            myw[lane] = make_double2(wa, wb);
        }
        __syncwarp();
        if (active) {
            const int64_t i0 = (int64_t)q * a.L + p0;
            double xv[V], yv[V];
            if (V == 2) {
                const double2 t = __ldg(reinterpret_cast<const double2 *>(x + i0));
                xv[0] = t.x;
                xv[V - 1] = t.y;
                if (ACCUM) {
                    const double2 u = __ldcs(reinterpret_cast<const double2 *>(y + i0));
                    yv[0] = u.x;
                    yv[V - 1] = u.y;
                }
            } else {
                xv[0] = __ldg(x + i0);
                if (ACCUM) yv[0] = __ldcs(y + i0);
            }
            double xg[NR][V];
#pragma unroll
            for (int r = 0; r < NR; ++r) {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    int64_t src = i0 + v - a.delta[r];
                    src = src < 0 ? 0 : (src > nm1 ? nm1 : src);
                    xg[r][v] = __ldg(x + src);
                }
            }
            double acc[V], dg[V];
#pragma unroll
            for (int v = 0; v < V; ++v) acc[v] = dg[v] = 0.0;
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const double2 w = myw[r];
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    dg[v] = fma(w.y, Fb[v][r], dg[v]);
                    acc[v] = fma(w.x * Fa[v][r], xg[r][v], acc[v]);
                }
            }
            double out[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                out[v] = fma(-dg[v], xv[v], acc[v]);
                if (ACCUM) out[v] += yv[v];
            }
            if (V == 2) {
                __stcs(reinterpret_cast<double2 *>(y + i0), make_double2(out[0], out[V - 1]));
            } else {
                __stcs(y + i0, out[0]);
            }
        }
        __syncwarp();
    }
}

struct KronData {
    int64_t n = 0;
    int ns = 0, nr = 0, k = 0, L = 0, Q = 0, V = 1, NR = 4, n_chunks = 1;
    int tab_stride = 0;
    double *d_tables = nullptr;
    int *d_nu = nullptr;
    std::vector<int> dims, tab_off, delta;
    int64_t halo = 0;
    int grid_full = 0;
};

using KronKernel = void (*)(const KronArgs, const double *, double *);

template <int NR, int V>
static KronKernel pick_accum(bool accum) {
    return accum ? k_kron_mv<NR, V, true> : k_kron_mv<NR, V, false>;
}

static KronKernel pick_kernel(int NR, int V, bool accum) {
    if (V == 2) {
        switch (NR) {
            case 4: return pick_accum<4, 2>(accum);
            case 8: return pick_accum<8, 2>(accum);
            case 12: return pick_accum<12, 2>(accum);
            case 16: return pick_accum<16, 2>(accum);
            default: return nullptr;
        }
    }
    switch (NR) {
        case 4: return pick_accum<4, 1>(accum);
        case 8: return pick_accum<8, 1>(accum);
        case 12: return pick_accum<12, 1>(accum);
        case 16: return pick_accum<16, 1>(accum);
        case 24: return pick_accum<24, 1>(accum);
        case 32: return pick_accum<32, 1>(accum);
        default: return nullptr;
    }
}

cufsp_status kron_create(const ModelHost &m, KronData **out) {
    if (m.nr > CUFSP_MAX_REACTIONS)
        return set_error(CUFSP_ERR_UNSUPPORTED, "KRONECKER format supports at most 32 reactions");
    KronData *kd = new KronData();
    kd->n = m.n;
    kd->ns = m.ns;
    kd->nr = m.nr;
    kd->tab_stride = m.tab_stride;
    kd->tab_off = m.tab_off;
    kd->dims.resize(m.ns);
    for (int s = 0; s < m.ns; ++s) kd->dims[s] = m.bounds[s] + 1;
    kd->NR = m.nr <= 4 ? 4 : m.nr <= 8 ? 8 : m.nr <= 12 ? 12 : m.nr <= 16 ? 16 : m.nr <= 24 ? 24 : 32;

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
        if (d > m.n || d < -m.n) d = 0;  // such a neighbour is never inside the box
        kd->delta[r] = (int)d;
        kd->halo = std::max<int64_t>(kd->halo, d < 0 ? -d : d);
    }

    // Occupancy-derived persistent grid (computed for the V=1 kernel; refined below).
    const DeviceInfo &di = device_info();
    // Inner split: choose k (species 0..k-1 inner) to minimise idle lanes in the last chunk.
    double best_waste = 1e30;
    int best_k = 1;
    int64_t Lk = 1;
    for (int k = 1; k <= m.ns; ++k) {
        Lk *= kd->dims[k - 1];
        if (Lk > 2147483647LL) break;
        const int Vk = (Lk % 2 == 0 && kd->NR <= 8) ? 2 : 1;
        const int64_t w = 32LL * Vk;
        const int64_t chunks = (Lk + w - 1) / w;
        if (chunks > (int64_t)di.sm_count * 16) break;  // keep at least ~4 rows of warps per sweep
        const double waste = (double)(chunks * w - Lk) / (double)Lk;
        if (waste < best_waste - 1e-12) {
            best_waste = waste;
            best_k = k;
        }
    }
    kd->k = best_k;
    int64_t L = 1;
    for (int s = 0; s < best_k; ++s) L *= kd->dims[s];
    kd->L = (int)L;
    kd->Q = (int)(m.n / L);
    kd->V = (L % 2 == 0 && kd->NR <= 8) ? 2 : 1;
    kd->n_chunks = (int)((L + 32LL * kd->V - 1) / (32LL * kd->V));

    int occ = 0;
    KronKernel kern = pick_kernel(kd->NR, kd->V, true);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, 0);
    if (e != cudaSuccess || occ < 1) occ = 1;
    kd->grid_full = di.sm_count * occ;

    const size_t tsz = (size_t)m.nr * m.tab_stride;
    e = cudaMalloc(&kd->d_tables, sizeof(double) * tsz);
    if (e == cudaSuccess) e = cudaMalloc(&kd->d_nu, sizeof(int) * m.nu.size());
    if (e == cudaSuccess) e = cudaMemcpy(kd->d_tables, m.tables.data(), sizeof(double) * tsz, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(kd->d_nu, m.nu.data(), sizeof(int) * m.nu.size(), cudaMemcpyHostToDevice);
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
    delete k;
}

int64_t kron_halo(const KronData *k) { return k->halo; }
int64_t kron_row_len(const KronData *k) { return k->L; }

cufsp_status kron_apply(KronData *kd, const double *coefs, double alpha, const double *d_alpha, const int *d_skip,
                        const double *x, bool accumulate, double *y, cudaStream_t st, int64_t i_begin, int64_t i_end) {
    KronArgs a;
    a.tables = kd->d_tables;
    a.nu = kd->d_nu;
    a.d_alpha = d_alpha;
    a.d_skip = d_skip;
    a.n = kd->n;
    a.tab_stride = kd->tab_stride;
    a.ns = kd->ns;
    a.nr = kd->nr;
    a.k = kd->k;
    a.L = kd->L;
    a.n_chunks = kd->n_chunks;
    if (i_end < 0) i_end = kd->n;
    a.q_begin = (int)(i_begin / kd->L);
    a.q_end = (int)((i_end + kd->L - 1) / kd->L);
    for (int s = 0; s < CUFSP_MAX_SPECIES; ++s) {
        a.dims[s] = s < kd->ns ? kd->dims[s] : 1;
        a.tab_off[s] = s < kd->ns ? kd->tab_off[s] : 0;
    }
    for (int r = 0; r < CUFSP_MAX_REACTIONS; ++r) {
        a.delta[r] = r < kd->nr ? kd->delta[r] : 0;
        a.coef[r] = r < kd->nr ? alpha * coefs[r] : 0.0;
    }
    const int rows = a.q_end - a.q_begin;
    if (rows <= 0) return CUFSP_SUCCESS;
    // Enough warps for every chunk, at most the persistent grid, and >= ~4 rows per warp.
    int64_t want_warps = (int64_t)kd->n_chunks * ((rows + 3) / 4);
    int64_t grid = (want_warps + 7) / 8;
    int64_t min_grid = (kd->n_chunks + 7) / 8;
    grid = std::max(grid, min_grid);
    grid = std::min<int64_t>(grid, std::max<int64_t>(kd->grid_full, min_grid));
    KronKernel kern = pick_kernel(kd->NR, kd->V, accumulate);
    if (!kern) return set_error(CUFSP_ERR_UNSUPPORTED, "no KRONECKER kernel for this reaction count");
    kern<<<(unsigned)grid, 256, 0, st>>>(a, x, y);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

}  // namespace cufsp
