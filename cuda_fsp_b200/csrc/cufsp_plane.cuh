// cufsp_plane.cuh -- KRONECKER generator action for near-neighbour networks, specialised per model.
//
// Same operator as k_kron_mv (cufsp_kron.cu) and the reference's fspmat_sdkron_mv
// (src/fspmat_kron_kernels.cu:51-129):
//   y[x] (+)= alpha * sum_r c_r ( a_r(x - nu_r) x[x - nu_r] 1{x - nu_r in box} - a_r(x) x[x] ),
//   a_r(x) = prod_s f_{r,s}(x_s),
// for boxes of 2 or 3 species whose reactions change every species by at most one molecule.
//
// This file is compiled at generator-create time by NVRTC, after a prefix (cufsp_kron_plane.cu)
// that fixes the reaction pattern as compile-time constants: per reaction its stoichiometry, its
// shifted and unshifted species-0 factor slots (identical tables share a slot; a table that is 1
// everywhere needs no register and no multiply), and the merged terms and diagonal groups built
// from them.  With the pattern fixed, every neighbour value is a named register.
//
// Layout and data flow (one CTA = one tile of TR rows x all n0 positions, marching over planes):
//  * species 0 runs along the lanes: lane l of warp c owns the pair x0 = 64 c + 2 l, 2 l + 1.
//    x0 +- 1 neighbours come from the lane itself or its neighbour lane by shuffle; lanes 0 / 31
//    take the value beyond their warp from shared memory ("edge").
//  * species 1 ("rows"): the tile rows plus one halo row above and below; with 2 species there
//    are no rows (TR = 1, no halo).
//  * species 2 ("planes") is the marching axis.  For every plane the tile rows of x, the tile rows
//    of y (accumulate form) and the tile's row words arrive by TMA bulk copies
//    (cp.async.bulk + mbarrier complete_tx) in a ring of S shared-memory stages, issued by one
//    thread up to S planes ahead.  Each thread moves its values of plane z + 1 from the ring into
//    a 3-plane register queue (z - 1, z, z + 1), so every x value crosses HBM once and shared
//    memory once, and is reused from registers for all 3^3 neighbour offsets.
//  * Row words (c_r x outer factor, merged per term / diagonal group) come from a table the host
//    rebuilds when the coefficients change (cufsp_kron_plane.cu), staged with the plane; one CTA
//    barrier per plane releases the stage.
//  * Every mbarrier wait is bounded.  On expiry the CTA records an error in *err, waits (bounded)
//    for its own copies still in flight, and returns; no CTA exits with a copy outstanding.
//  * Rows outside the box are never copied: their stage rows are zeroed once and their
//    coefficients are zero.  Planes outside the box copy the nearest plane (finite values that
//    meet zero coefficients).
// x and y must be 16-byte aligned and n0 even (pairs); the host checks both.

#ifndef CUFSP_PLANE_CUH
#define CUFSP_PLANE_CUH

#ifndef CUFSP_PLANE_MAX_R
#define CUFSP_PLANE_MAX_R 32
#endif

struct CufspPlaneArgs {
    const double *words;   // [n1 * n2][nwp] row words: c_r x outer factors, merged per term / group
    const double *tab0;    // species-0 factor tables, tab0[r * tab_stride + x0]
    const double *d_alpha; // nullable device scalar multiplying every coefficient
    const int *d_skip;     // nullable: return at once when *d_skip != 0
    int *err;              // watchdog flag: set when a bounded barrier wait expired
    int n0, n1, n2;        // box extents (n1 = 1 with 2 species)
    int tab_stride;
    int pitch;             // doubles per staged row (n0 rounded up to 64)
    int row_blocks;        // n1 / TR
    int zseg;              // planes per segment
    int z_begin, z_end;    // planes to compute
    int items;             // row_blocks * segments = CTAs
    int nwp;               // words per row, padded to even
    double alpha;          // scale of every coefficient (times *d_alpha)
};

#ifdef __CUDACC_RTC__

namespace cufsp_plane {

constexpr int NR = CUFSP_PLANE_NR;      // reactions
constexpr int NOFF = CUFSP_PLANE_NOFF;  // distinct neighbour offsets
constexpr int NFA = CUFSP_PLANE_NFA;    // shifted species-0 factor slots held in registers
constexpr int NFB = CUFSP_PLANE_NFB;    // unshifted species-0 factor slots held in registers
constexpr int NT = CUFSP_PLANE_NT;      // shifted terms (offset, factor slot)
constexpr int NDG = CUFSP_PLANE_NDG;    // diagonal groups (factor slot or constant 1)
constexpr int TR = CUFSP_PLANE_TR;      // tile rows
constexpr int S = CUFSP_PLANE_STAGES;   // ring stages
constexpr int PPS = CUFSP_PLANE_PPS;    // planes per CTA barrier (1 or 2)
static_assert(PPS == 1 || (PPS == 2 && S >= 4), "two planes per step need at least 4 stages");
constexpr bool ROWS = CUFSP_PLANE_ROWS != 0;
constexpr bool YTMA = CUFSP_PLANE_YTMA != 0;  // stage y rows in the ring (else L2 prefetch + loads)
constexpr int NQ = ROWS ? TR + 2 : 1;   // staged x rows per plane (tile + halo)
constexpr int NW = NT + NDG;            // row words per tile row
constexpr int NWP = (NW + 1) & ~1;      // padded to a 16-byte multiple
constexpr int NFA1 = NFA > 0 ? NFA : 1;
constexpr int NFB1 = NFB > 0 ? NFB : 1;

// The generated prefix defines, in this namespace, constexpr functions of a constant index:
//   nu0(r)                 net change of reaction r in species 0
//   o0(k), o1(k), o2(k)    net change of distinct offset k in species 0, 1, 2 (source x - o)
//   t_off(t), t_fa(t)      offset and shifted factor slot (-1: constant 1) of term t
//   r_term(r), r_dg(r)     term and diagonal group of reaction r
//   fa_rep(s), fb_rep(s)   a reaction whose table defines register slot s
//   dg_fb(g)               unshifted factor slot of diagonal group g (-1: constant 1)

// ---- bounded TMA / mbarrier helpers ------------------------------------------------------------
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
// Each try_wait suspends for a hardware-defined interval; false after `tries` tries.  The waits
// before a plane is computed use CUFSP_PLANE_WAIT_TRIES (2^20 unless the host asks for fewer, which
// only the watchdog's own test does: 0 makes every such wait give up at once); the final drain of
// copies still in flight always uses 2^20, so no CTA leaves with a copy outstanding.
#ifndef CUFSP_PLANE_WAIT_TRIES
#define CUFSP_PLANE_WAIT_TRIES (1 << 20)
#endif
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
__device__ __forceinline__ void prefetch_l2_bulk(const void *src, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Stage layout (doubles): x rows [NQ][pitch], y rows [YR][pitch], row words [TR][NWP].
template <bool ACCUM>
struct Layout {
    static constexpr int YR = (ACCUM && YTMA) ? TR : 0;
    __device__ static int doubles(int pitch) { return (NQ + YR) * pitch + TR * NWP; }
    __device__ static int y_off(int pitch) { return NQ * pitch; }
    __device__ static int g_off(int pitch) { return (NQ + YR) * pitch; }
};

struct Tile {
    int x1_0;      // first tile row
    int rlo, rhi;  // staged x rows [rlo, rhi) of the NQ (rows inside the box)
    int z0, z1;    // output planes [z0, z1)
};

// Issue the copies of plane p into its stage (one thread).
template <bool ACCUM>
__device__ __forceinline__ void issue_plane(const CufspPlaneArgs &a, const Tile &t, const double *x, const double *y,
                                            double *stage, unsigned long long *bar, int p) {
    const int pc = min(max(p, 0), a.n2 - 1);
    const bool out = p >= t.z0 && p < t.z1;
    const unsigned row_bytes = (unsigned)a.n0 * 8u;
    unsigned bytes = (unsigned)(t.rhi - t.rlo) * row_bytes;
    if (out) bytes += (unsigned)Layout<ACCUM>::YR * row_bytes + (unsigned)(TR * NWP * 8);
    mbar_expect_tx(bar, bytes);
    const size_t plane = (size_t)pc * a.n1;
    for (int i = t.rlo; i < t.rhi; ++i) {
        const int x1 = ROWS ? t.x1_0 - 1 + i : 0;
        tma_load(stage + i * a.pitch, x + (plane + x1) * a.n0, row_bytes, bar);
    }
    if (out) {
        for (int j = 0; j < Layout<ACCUM>::YR; ++j)
            tma_load(stage + Layout<ACCUM>::y_off(a.pitch) + j * a.pitch, y + (plane + t.x1_0 + j) * a.n0, row_bytes,
                     bar);
        if (ACCUM && !YTMA)
            for (int j = 0; j < TR; ++j) prefetch_l2_bulk(y + (plane + t.x1_0 + j) * a.n0, row_bytes);
        const size_t q = (size_t)(ROWS ? t.x1_0 : 0) + (size_t)a.n1 * p;
        tma_load(stage + Layout<ACCUM>::g_off(a.pitch), a.words + q * NWP, (unsigned)(TR * NWP * 8), bar);
    }
}

struct Lane {
    int lane, warp, x0;
    bool active, has_left, has_right;
};

// Queue slot: the lane's pair of every staged row of one plane, and its edge value per row.
struct Slot {
    double2 q[NQ];
    double e[NQ];
};

__device__ __forceinline__ void load_slot(const Lane &L, const double *stage, int pitch, Slot &s) {
    const int c0 = L.warp * 64;
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const double *row = stage + i * pitch;
        s.q[i] = *reinterpret_cast<const double2 *>(row + L.x0);
        double e = 0.0;
        if (L.lane == 0 && L.has_left) e = row[c0 - 1];
        if (L.lane == 31 && L.has_right) e = row[c0 + 64];
        s.e[i] = e;
    }
}

// Neighbour pair x[x0 - d0 .. x0 + 1 - d0] of a queued row, d0 = net change in species 0.
template <int D0>
__device__ __forceinline__ double2 shifted(const Lane &L, double2 q, double e) {
    if constexpr (D0 == 0) {
        return q;
    } else if constexpr (D0 == 1) {  // source x0 - 1
        const double left = __shfl_up_sync(0xffffffffu, q.y, 1);
        return make_double2(L.lane == 0 ? e : left, q.x);
    } else {  // source x0 + 1
        const double right = __shfl_down_sync(0xffffffffu, q.x, 1);
        return make_double2(q.y, L.lane == 31 ? e : right);
    }
}

// Neighbour values of tile row J for offsets K.. (recursion keeps every index a constant).
template <int J, int K>
__device__ __forceinline__ void fill_offsets(const Lane &L, const Slot &sm, const Slot &s0, const Slot &sp,
                                             double2 (&v)[NOFF]) {
    if constexpr (K < NOFF) {
        constexpr int qi = ROWS ? J - o1(K) + 1 : 0;
        if constexpr (o2(K) == 1) v[K] = shifted<o0(K)>(L, sm.q[qi], sm.e[qi]);
        else if constexpr (o2(K) == 0) v[K] = shifted<o0(K)>(L, s0.q[qi], s0.e[qi]);
        else v[K] = shifted<o0(K)>(L, sp.q[qi], sp.e[qi]);
        fill_offsets<J, K + 1>(L, sm, s0, sp, v);
    }
}

// Output pair of tile row J of plane z.
template <bool ACCUM, int J>
__device__ __forceinline__ void compute_row(const CufspPlaneArgs &a, const Lane &L, const Tile &t, int z,
                                            const Slot &sm, const Slot &s0, const Slot &sp, const double *words,
                                            const double *ystage, const double (&Fa)[2][NFA1],
                                            const double (&Fb)[2][NFB1], double alpha, double *__restrict__ y) {
    double *yp = y + ((size_t)z * a.n1 + (ROWS ? t.x1_0 + J : 0)) * a.n0 + L.x0;
    double2 yv = make_double2(0.0, 0.0);
    if constexpr (ACCUM) {
        if constexpr (YTMA) yv = *reinterpret_cast<const double2 *>(ystage + J * a.pitch + L.x0);
        else if (L.active) yv = __ldcs(reinterpret_cast<const double2 *>(yp));
    }
    double w[NWP];
#pragma unroll
    for (int k = 0; k < NWP; k += 2) {
        const double2 wp = *reinterpret_cast<const double2 *>(words + J * NWP + k);
        w[k] = wp.x;
        w[k + 1] = wp.y;
    }
    double2 v[NOFF];
    fill_offsets<J, 0>(L, sm, s0, sp, v);
    double a0[2] = {0.0, 0.0}, a1[2] = {0.0, 0.0};  // two partial sums per position (ILP)
#pragma unroll
    for (int tt = 0; tt < NT; ++tt) {
        const double2 val = v[t_off(tt)];
        const int sl = t_fa(tt);
        const double w0 = sl < 0 ? w[tt] : w[tt] * Fa[0][sl < 0 ? 0 : sl];
        const double w1 = sl < 0 ? w[tt] : w[tt] * Fa[1][sl < 0 ? 0 : sl];
        a0[tt & 1] = fma(w0, val.x, a0[tt & 1]);
        a1[tt & 1] = fma(w1, val.y, a1[tt & 1]);
    }
    double d0 = 0.0, d1 = 0.0;
#pragma unroll
    for (int g = 0; g < NDG; ++g) {
        const int sl = dg_fb(g);
        d0 = sl < 0 ? d0 + w[NT + g] : fma(w[NT + g], Fb[0][sl < 0 ? 0 : sl], d0);
        d1 = sl < 0 ? d1 + w[NT + g] : fma(w[NT + g], Fb[1][sl < 0 ? 0 : sl], d1);
    }
    const double2 c = s0.q[ROWS ? J + 1 : 0];
    double o0v = alpha * fma(-d0, c.x, a0[0] + a0[1]);
    double o1v = alpha * fma(-d1, c.y, a1[0] + a1[1]);
    if constexpr (ACCUM) {
        o0v += yv.x;
        o1v += yv.y;
    }
    if (L.active) __stcs(reinterpret_cast<double2 *>(yp), make_double2(o0v, o1v));
}

template <bool ACCUM, int J>
__device__ __forceinline__ void compute_rows(const CufspPlaneArgs &a, const Lane &L, const Tile &t, int z,
                                             const Slot &sm, const Slot &s0, const Slot &sp, const double *words,
                                             const double *ystage, const double (&Fa)[2][NFA1],
                                             const double (&Fb)[2][NFB1], double alpha, double *__restrict__ y) {
    if constexpr (J < TR) {
        compute_row<ACCUM, J>(a, L, t, z, sm, s0, sp, words, ystage, Fa, Fb, alpha, y);
        compute_rows<ACCUM, J + 1>(a, L, t, z, sm, s0, sp, words, ystage, Fa, Fb, alpha, y);
    }
}

template <bool ACCUM>
__device__ __forceinline__ void plane_mv(const CufspPlaneArgs &a, const double *__restrict__ x, double *__restrict__ y) {
    using LY = Layout<ACCUM>;
    extern __shared__ __align__(128) double smem[];
    __shared__ __align__(8) unsigned long long bars[S];
    __shared__ int failed_flag;
    if (a.d_skip && *a.d_skip) return;
    if ((int)blockIdx.x >= a.items) return;
    const int tid = threadIdx.x;
    Lane L;
    L.lane = tid & 31;
    L.warp = tid >> 5;
    L.x0 = L.warp * 64 + 2 * L.lane;
    L.active = L.x0 < a.n0;
    L.has_left = L.warp > 0;
    L.has_right = L.warp * 64 + 64 < a.n0;
    Tile t;
    const int rb = blockIdx.x % a.row_blocks, seg = blockIdx.x / a.row_blocks;
    t.x1_0 = rb * TR;
    t.z0 = a.z_begin + seg * a.zseg;
    t.z1 = min(a.z_end, t.z0 + a.zseg);
    if (t.z0 >= t.z1) return;  // whole CTA leaves before any barrier or copy
    t.rlo = ROWS ? max(0, 1 - t.x1_0) : 0;
    t.rhi = ROWS ? min(NQ, a.n1 - t.x1_0 + 1) : 1;
    const int sd = LY::doubles(a.pitch);

    // zero every stage once (rows outside the box and the padding of short rows stay zero)
    for (int i = tid; i < S * sd; i += blockDim.x) smem[i] = 0.0;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) mbar_init(bars + s, 1);
        fence_mbar_init();
        failed_flag = 0;
    }
    fence_proxy_async();
    __syncthreads();

    // Planes p >= z0 - 1 map to stage (p - z0 + 1) % S with parity ((p - z0 + 1) / S) & 1.
    const int pbase = t.z0 - 1;
    const int p_last = t.z1;  // the halo plane after the segment is the last one read
    int issued = pbase - 1;
    if (tid == 0) {
        const int stop = min(p_last, pbase + S - 1);
        for (int p = pbase; p <= stop; ++p)
            issue_plane<ACCUM>(a, t, x, y, smem + ((p - pbase) % S) * sd, bars + (p - pbase) % S, p);
        issued = stop;
    }

    // inner factors of the lane's two positions (registers, fixed for the launch)
    double Fa[2][NFA1], Fb[2][NFB1];
#pragma unroll
    for (int v = 0; v < 2; ++v) {
        const int xv = L.active ? L.x0 + v : 0;
#pragma unroll
        for (int s = 0; s < NFA1; ++s) {
            Fa[v][s] = 1.0;
            if (s < NFA) {
                const int r = fa_rep(s), xs = xv - nu0(r);
                Fa[v][s] = (xs < 0 || xs >= a.n0) ? 0.0 : __ldg(a.tab0 + r * a.tab_stride + xs);
            }
        }
#pragma unroll
        for (int s = 0; s < NFB1; ++s) Fb[v][s] = s < NFB ? __ldg(a.tab0 + fb_rep(s) * a.tab_stride + xv) : 1.0;
    }
    const double alpha = a.alpha * (a.d_alpha ? __ldg(a.d_alpha) : 1.0);

    auto stage_of = [&](int p) { return smem + ((p - pbase) % S) * sd; };
    auto wait_plane = [&](int p) -> bool {
        return mbar_wait_bounded(bars + (p - pbase) % S, ((p - pbase) / S) & 1, CUFSP_PLANE_WAIT_TRIES);
    };
    auto drain_plane = [&](int p) -> bool {
        return mbar_wait_bounded(bars + (p - pbase) % S, ((p - pbase) / S) & 1, 1 << 20);
    };

    bool bad = false;
    Slot q0, q1, q2, q3;
    // prologue: planes z0 - 1 and z0 into the queue
    if (wait_plane(pbase) && wait_plane(t.z0)) {
        load_slot(L, stage_of(pbase), a.pitch, PPS == 1 ? q2 : q3);
        load_slot(L, stage_of(t.z0), a.pitch, q0);
    } else {
        failed_flag = 1;
    }
    __syncthreads();
    bad = failed_flag != 0;
    const bool prologue_ok = !bad;

    int z = t.z0;
    // Refill after a CTA barrier: every stage whose plane the CTA has finished with goes to the next
    // plane at once -- after the prologue the halo plane z0 - 1, after step z plane z (its x rows went
    // into the register queue one step earlier, its y rows and words were used in step z).
    auto refill = [&](int count) {
        if (tid == 0)
            for (int k = 0; k < count && issued < p_last; ++k) {
                ++issued;
                fence_proxy_async();
                issue_plane<ACCUM>(a, t, x, y, stage_of(issued), bars + (issued - pbase) % S, issued);
            }
    };
    if (!bad) refill(1);
    if constexpr (PPS == 1) {
        // Step z: the slots hold (z - 1, z, z + 1) in a fixed rotation of 3; one barrier per plane.
        auto step = [&](Slot &sm, Slot &s0, Slot &sp) -> bool {
            if (bad || z >= t.z1) return false;
            if (wait_plane(z + 1)) {
                load_slot(L, stage_of(z + 1), a.pitch, sp);
                const double *st = stage_of(z);
                compute_rows<ACCUM, 0>(a, L, t, z, sm, s0, sp, st + LY::g_off(a.pitch), st + LY::y_off(a.pitch), Fa,
                                       Fb, alpha, y);
            } else {
                failed_flag = 1;
            }
            __syncthreads();  // the stage of z is consumed
            if (failed_flag) {
                bad = true;
                return false;
            }
            refill(1);
            ++z;
            return true;
        };
        while (step(q2, q0, q1) && step(q0, q1, q2) && step(q1, q2, q0)) {
        }
    } else {
        // Double step z: slots (z - 1, z, z + 1, z + 2) in a rotation of 4; planes z and z + 1 are
        // computed under one barrier (z + 1 only while inside the segment).
        auto step2 = [&](Slot &sa, Slot &sb, Slot &sc, Slot &sd) -> bool {
            if (bad || z >= t.z1) return false;
            const bool two = z + 1 < t.z1;
            if (wait_plane(z + 1) && (!two || wait_plane(z + 2))) {
                load_slot(L, stage_of(z + 1), a.pitch, sc);
                if (two) load_slot(L, stage_of(z + 2), a.pitch, sd);
                const double *st = stage_of(z);
                compute_rows<ACCUM, 0>(a, L, t, z, sa, sb, sc, st + LY::g_off(a.pitch), st + LY::y_off(a.pitch), Fa,
                                       Fb, alpha, y);
                if (two) {
                    const double *st1 = stage_of(z + 1);
                    compute_rows<ACCUM, 0>(a, L, t, z + 1, sb, sc, sd, st1 + LY::g_off(a.pitch),
                                           st1 + LY::y_off(a.pitch), Fa, Fb, alpha, y);
                }
            } else {
                failed_flag = 1;
            }
            __syncthreads();  // the stages of z and z + 1 are consumed
            if (failed_flag) {
                bad = true;
                return false;
            }
            refill(two ? 2 : 1);
            z += two ? 2 : 1;
            return true;
        };
        while (step2(q3, q0, q1, q2) && step2(q1, q2, q3, q0)) {
        }
    }
    if (tid == 0) {
        // every issued copy must have landed before the CTA's shared memory is released: after a
        // failed prologue none was waited for; otherwise the planes up to z were
        for (int p = prologue_ok ? z + 1 : pbase; p <= issued; ++p)
            if (!drain_plane(p)) bad = true;
        if (bad) atomicExch(a.err, 1);
    }
}

}  // namespace cufsp_plane

extern "C" __global__ void __launch_bounds__(CUFSP_PLANE_THREADS, CUFSP_PLANE_MINB)
    cufsp_plane_mv_accum(const CufspPlaneArgs a, const double *__restrict__ x, double *__restrict__ y) {
    cufsp_plane::plane_mv<true>(a, x, y);
}

extern "C" __global__ void __launch_bounds__(CUFSP_PLANE_THREADS, CUFSP_PLANE_MINB)
    cufsp_plane_mv_set(const CufspPlaneArgs a, const double *__restrict__ x, double *__restrict__ y) {
    cufsp_plane::plane_mv<false>(a, x, y);
}

#endif  // __CUDACC_RTC__
#endif  // CUFSP_PLANE_CUH
