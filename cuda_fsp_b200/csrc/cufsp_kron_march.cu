// cufsp_kron_march.cu -- KRONECKER generator action, TMA-fed marching kernel (fast path).
//
// Same operator as k_kron_mv (cufsp_kron.cu), organised for data reuse inside one SM:
//  * The slowest species is the marching axis z; a "plane" is all states with one value of it
//    (P = n / n_z states).  Inside a plane, states form rows of L inner positions.
//  * A CTA owns a tile of R consecutive rows (full rows: W warps x 32 lanes x V positions = L) and
//    marches over a segment of planes.  For every plane it reads, the tile rows plus the halo rows
//    reached by in-plane row shifts arrive as ONE contiguous TMA bulk copy
//    (cp.async.bulk ... mbarrier::complete_tx) into a ring of plane slots in shared memory.  Plane
//    shifts (nu_z != 0) read neighbouring slots; every gather x[i - d_r] is a shared-memory load,
//    so x crosses L2 about once per tile (plus halo rows) instead of once per gather.
//  * Each lane keeps the inner factor products of its fixed positions in registers (as k_kron_mv);
//    the row-uniform outer factors G(q) come from the create-time table, multiplied by c_r once per
//    tile row and plane into shared memory.
//  * Copies are issued in plane order by one thread, at most `slots` planes ahead; every mbarrier
//    wait is bounded.  On expiry the CTA records an error in *err, waits (bounded) for its own
//    copies still in flight, and returns.  No CTA exits with a copy outstanding.
// Slots carry guard elements on both sides so that shifted in-row reads of invalid neighbours
// (coefficient 0) stay inside the slot; slot memory is zeroed once, so such reads are finite.
#include <algorithm>
#include <cstdint>

#include "cufsp_internal.h"
#include "cufsp_march.h"

namespace cufsp {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait (each try_wait itself suspends for a hardware-defined interval); false on expiry.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
    for (int it = 0; it < (1 << 20); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_1d(void *dst_smem, const void *src_gmem, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst_smem)),
                 "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Planes zp >= z0 map to slot (zp - z0) % slots, phase (zp - z0) / slots.
struct Ring {
    int z0, slots;
    __device__ __forceinline__ int slot(int zp) const { return (zp - z0) % slots; }
    __device__ __forceinline__ uint32_t parity(int zp) const { return (uint32_t)(((zp - z0) / slots) & 1); }
};

// Issue the copy of plane zp (tile rows [r0 - hr_lo, r0 + R + hr_hi) clipped to the plane) into its
// slot; planes outside [0, Z) only arrive on their barrier.  One thread.
__device__ __forceinline__ void march_issue(const MarchArgs &a, const double *__restrict__ x, double *ring,
                                            uint64_t *bars, const Ring &rg, int zp, int r0) {
    const int s = rg.slot(zp);
    uint64_t *bar = bars + s;
    if (zp < 0 || zp >= a.Z) {
        mbar_expect_tx(bar, 0);
        return;
    }
    const int rlo = max(r0 - a.hr_lo, 0);
    const int rhi = min(r0 + a.R + a.hr_hi, a.RP);
    const uint32_t bytes = (uint32_t)(rhi - rlo) * (uint32_t)a.L * 8u;
    mbar_expect_tx(bar, bytes);
    if (bytes) {
        double *dst = ring + (size_t)s * a.slot_elems + a.guard + (size_t)(rlo - (r0 - a.hr_lo)) * a.L;
        const double *src = x + (size_t)zp * a.P + (size_t)rlo * a.L;
        tma_load_1d(dst, src, bytes, bar);
    }
}

#ifndef CUFSP_MARCH_MINB
#define CUFSP_MARCH_MINB 2
#endif
template <int NR, int V, bool ACCUM>
__global__ void __launch_bounds__(256, CUFSP_MARCH_MINB) k_kron_march(const MarchArgs a, const double *__restrict__ x,
                                                   double *__restrict__ y) {
    extern __shared__ __align__(128) double sm_dyn[];
    __shared__ __align__(8) uint64_t bars[kMarchMaxSlots];
    if (a.d_skip && *a.d_skip) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double *ring = sm_dyn;
    double2 *wtab = reinterpret_cast<double2 *>(ring + (size_t)a.slots * a.slot_elems);  // [R][NR]

    const int tile = blockIdx.x % a.row_tiles;
    const int zsegi = blockIdx.x / a.row_tiles;
    const int r0 = tile * a.R;
    const int z_begin = zsegi * a.zseg;
    const int z_end = min(a.Z, z_begin + a.zseg);
    const int rows = min(a.R, a.RP - r0);
    if (z_begin >= a.Z || rows <= 0) return;  // whole CTA leaves before any barrier or copy

    // zero the ring (guards and clipped rows must read as finite), then set up the barriers
    for (int i = tid; i < a.slots * a.slot_elems; i += blockDim.x) ring[i] = 0.0;
    if (tid == 0) {
        for (int s = 0; s < a.slots; ++s) mbar_init(bars + s, 1);
        fence_mbar_init();
    }
    fence_proxy_async_smem();
    __syncthreads();

    // inner factors of this lane's fixed positions p = warp * 32V + lane * V + v
    const int p0 = warp * (32 * V) + lane * V;
    double Fa[V][NR], Fb[V][NR];
#pragma unroll
    for (int v = 0; v < V; ++v) {
#pragma unroll
        for (int r = 0; r < NR; ++r) Fa[v][r] = Fb[v][r] = 1.0;
        int rem = p0 + v;
        for (int s = 0; s < a.k; ++s) {
            const int d = a.dims[s];
            const int xs = rem % d;
            rem /= d;
            const double *t = a.tables + a.tab_off[s];
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const double *tr = t + r * a.tab_stride;
                Fb[v][r] *= __ldg(tr + xs);
                const int xsh = xs - __ldg(a.nu + r * a.ns + s);
                Fa[v][r] = (xsh < 0 || xsh >= d) ? 0.0 : Fa[v][r] * __ldg(tr + xsh);
            }
        }
    }
    const double alpha_dev = a.d_alpha ? __ldg(a.d_alpha) : 1.0;

    const Ring rg{z_begin - a.hz_lo, a.slots};
    const int z_last = z_end - 1 + a.hz_hi;  // last plane any step of this segment reads
    int issued = rg.z0 - 1;                  // planes rg.z0 .. issued have been issued (thread 0's view)
    if (tid == 0) {
        const int stop = min(z_last, rg.z0 + a.slots - 1);
        for (int zp = rg.z0; zp <= stop; ++zp) march_issue(a, x, ring, bars, rg, zp, r0);
        issued = stop;
    }
    int waited = rg.z0 - 1;  // planes up to `waited` are complete (every thread's view)
    bool failed = false;
    // Software pipeline for the two global streams left in the loop: y of the next plane is
    // loaded right after each tile row is consumed, and the outer-factor entry (one per thread,
    // rows * NR <= blockDim) of the next plane is fetched one step ahead.
    const int gt = tid < rows * NR ? tid : -1;
    const int gj = gt >= 0 ? gt / NR : 0, gr = gt >= 0 ? gt - gj * NR : 0;
    double2 gpre = make_double2(0.0, 0.0);
    if (gt >= 0) gpre = __ldg(a.gtab + ((size_t)z_begin * a.RP + r0 + gj) * NR + gr);
    double ypre[kMarchMaxR][V];
#pragma unroll
    for (int j = 0; j < kMarchMaxR; ++j)
#pragma unroll
        for (int v = 0; v < V; ++v)
            ypre[j][v] = (ACCUM && j < rows) ? __ldcs(y + (size_t)z_begin * a.P + (size_t)(r0 + j) * a.L + p0 + v) : 0.0;
    for (int z = z_begin; z < z_end; ++z) {
        for (int zw = waited + 1; zw <= z + a.hz_hi && !failed; ++zw) {
            if (mbar_wait_bounded(bars + rg.slot(zw), rg.parity(zw))) waited = zw;
            else failed = true;
        }
        if (__syncthreads_or(failed)) break;
        // row-uniform outer factors for the tile rows at plane z
        if (gt >= 0) {
            const double c = a.coef[gr] * alpha_dev;
            wtab[gj * NR + gr] = make_double2(c * gpre.x, c * gpre.y);
            if (z + 1 < z_end) gpre = __ldg(a.gtab + ((size_t)(z + 1) * a.RP + r0 + gj) * NR + gr);
        }
        __syncthreads();
        const double *slotp[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) slotp[r] = ring + (size_t)rg.slot(z - a.dz[r]) * a.slot_elems + a.guard + a.soff[r];
        const double *cen = ring + (size_t)rg.slot(z) * a.slot_elems + a.guard + (size_t)a.hr_lo * a.L;
        const size_t zbase = (size_t)z * a.P + (size_t)r0 * a.L;
        const bool more = z + 1 < z_end;
#pragma unroll
        for (int j = 0; j < kMarchMaxR; ++j) {
            if (j >= rows) break;
            const int e = j * a.L + p0;
            double yv[V];
#pragma unroll
            for (int v = 0; v < V; ++v) yv[v] = ypre[j][v];
            if (ACCUM && more) {
#pragma unroll
                for (int v = 0; v < V; ++v) ypre[j][v] = __ldcs(y + zbase + a.P + e + v);
            }
            double acc[V], dg[V], xv[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                acc[v] = dg[v] = 0.0;
                xv[v] = cen[e + v];
            }
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const double2 w = wtab[j * NR + r];
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    dg[v] = fma(w.y, Fb[v][r], dg[v]);
                    acc[v] = fma(w.x * Fa[v][r], slotp[r][e + v], acc[v]);
                }
            }
#pragma unroll
            for (int v = 0; v < V; ++v) {
                double o = fma(-dg[v], xv[v], acc[v]);
                if (ACCUM) o += yv[v];
                __stcs(y + zbase + e + v, o);
            }
        }
        __syncthreads();  // all reads of plane z - hz_lo's slot are done: it may be refilled
        if (tid == 0 && issued < z_last) {
            fence_proxy_async_smem();
            ++issued;
            march_issue(a, x, ring, bars, rg, issued, r0);
        }
    }
    if (tid == 0) {
        // every issued copy must have landed before the CTA's shared memory is released
        for (int zw = waited + 1; zw <= issued; ++zw)
            if (!mbar_wait_bounded(bars + rg.slot(zw), rg.parity(zw))) failed = true;
        if (failed) atomicExch(a.err, 1);
    }
}

#define MARCH_CASE(NRv, Vv) \
    case NRv:               \
        return accum ? (MarchKernel)k_kron_march<NRv, Vv, true> : (MarchKernel)k_kron_march<NRv, Vv, false>;

MarchKernel pick_march_kernel(int NR, int V, bool accum) {
    if (V == 2) {
        switch (NR) {
            MARCH_CASE(1, 2) MARCH_CASE(2, 2) MARCH_CASE(3, 2) MARCH_CASE(4, 2) MARCH_CASE(5, 2) MARCH_CASE(6, 2)
            MARCH_CASE(7, 2) MARCH_CASE(8, 2) MARCH_CASE(9, 2) MARCH_CASE(10, 2) MARCH_CASE(11, 2) MARCH_CASE(12, 2)
            default: return nullptr;
        }
    }
    if (V == 1) {
        switch (NR) {
            MARCH_CASE(1, 1) MARCH_CASE(2, 1) MARCH_CASE(3, 1) MARCH_CASE(4, 1) MARCH_CASE(5, 1) MARCH_CASE(6, 1)
            MARCH_CASE(7, 1) MARCH_CASE(8, 1) MARCH_CASE(9, 1) MARCH_CASE(10, 1) MARCH_CASE(11, 1) MARCH_CASE(12, 1)
            MARCH_CASE(13, 1) MARCH_CASE(14, 1) MARCH_CASE(15, 1) MARCH_CASE(16, 1)
            default: return nullptr;
        }
    }
    return nullptr;
}
#undef MARCH_CASE

}  // namespace cufsp
