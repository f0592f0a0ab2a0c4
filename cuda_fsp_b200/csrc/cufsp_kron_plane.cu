// cufsp_kron_plane.cu -- host side of the runtime-specialised KRONECKER kernel (cufsp_plane.cuh).
//
// At generator-create time the reaction network is checked for the near-neighbour shape the plane
// kernel handles (2 or 3 species, every |nu_{r,s}| <= 1, an even species-0 extent up to 1024), its
// pattern -- distinct neighbour offsets, species-0 factor slots (identical tables shared, tables
// equal to 1 dropped), the shifted terms and diagonal groups built from them -- is written as a
// source prefix, and the kernel is compiled for sm_100a with NVRTC and loaded with
// cudaLibraryLoadData.  Compiled kernels are cached per process by their full source text, so
// generators of the same network over other boxes reuse them.  Networks of other shapes, and
// applies over a range that is not whole planes, use k_kron_mv (cufsp_kron.cu).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>

#include "cufsp_internal.h"
#include "cufsp_plane.cuh"

namespace cufsp {

namespace {

const char *kPlaneSource =
#include "cufsp_plane_src.inc"
    ;

int env_int(const char *name, int dflt) {
    const char *v = getenv(name);
    return v ? atoi(v) : dflt;
}

void emit_fn(std::ostringstream &s, const char *name, const std::vector<int> &v) {
    s << "__host__ __device__ __forceinline__ constexpr int " << name << "(int i) {";
    for (size_t i = 0; i < v.size(); ++i) s << " if (i == " << i << ") return " << v[i] << ";";
    s << " return 0; }\n";
}

}  // namespace

// Row words of the plane kernel for one coefficient vector: for every row q of the outer index,
//   words[q][t]      = sum_{r in term t} c_r Ga_r(q)        (shifted terms)
//   words[q][nt + g] = sum_{r in group g} c_r Gb_r(q)       (diagonal groups), 0 in the padding,
// summed in reaction order (deterministic).
struct WordArgs {
    int nr, nt, nw, nwp;
    int r_term[CUFSP_PLANE_MAX_R], r_dg[CUFSP_PLANE_MAX_R];
    double coef[CUFSP_PLANE_MAX_R];
};

__global__ void k_plane_words(const WordArgs a, const double2 *__restrict__ gtab, int64_t rows, double *__restrict__ words) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * a.nwp) return;
    const int64_t q = i / a.nwp;
    const int k = (int)(i - q * a.nwp);
    double s = 0.0;
    for (int r = 0; r < a.nr; ++r) {
        const double2 g = gtab[q * a.nr + r];
        if (k < a.nt) {
            if (a.r_term[r] == k) s = fma(a.coef[r], g.x, s);
        } else if (k < a.nw && a.r_dg[r] == k - a.nt) {
            s = fma(a.coef[r], g.y, s);
        }
    }
    words[i] = s;
}

struct PlaneData {
    std::shared_ptr<RtcModule> k;  // kernels[0] accumulate form, kernels[1] overwrite form
    int n0 = 0, n1 = 1, n2 = 0, nr = 0, tr = 1;
    int row_blocks = 0, threads = 0, pitch = 0;
    size_t smem_accum = 0, smem_set = 0;
    int occ_accum = 1, occ_set = 1;
    int tab_stride = 0;
    double2 *d_gtab = nullptr;       // outer factors for the species-0 / rest split
    const double *d_tab0 = nullptr;  // species-0 tables inside the generator's table array
    int *h_err = nullptr, *d_err = nullptr;  // watchdog word of the bounded barrier waits (mapped host memory)
    double *d_words = nullptr;       // row words for the coefficients in words_coefs
    std::vector<double> words_coefs;
    WordArgs wa;
    std::string description;
};

namespace {

// Index of v in list (appended when new).
template <class T>
int intern(std::vector<T> &list, const T &v) {
    for (size_t i = 0; i < list.size(); ++i)
        if (list[i] == v) return (int)i;
    list.push_back(v);
    return (int)list.size() - 1;
}

bool all_ones(const std::vector<double> &v) {
    for (double d : v)
        if (d != 1.0) return false;
    return true;
}

}  // namespace

PlaneData *plane_create(const ModelHost &m, const double *d_tables, std::string &why) {
    why.clear();
    if (env_int("CUFSP_PLANE", 1) == 0) {
        why = "disabled (CUFSP_PLANE=0)";
        return nullptr;
    }
    if (m.ns < 2 || m.ns > 3) {
        why = "needs 2 or 3 species";
        return nullptr;
    }
    if (m.nr > CUFSP_PLANE_MAX_R) {
        why = "more than 32 reactions";
        return nullptr;
    }
    for (int v : m.nu)
        if (v < -1 || v > 1) {
            why = "a reaction changes a species by more than one";
            return nullptr;
        }
    const int n0 = m.bounds[0] + 1;
    if (n0 % 2 != 0) {
        why = "species 0 extent is odd";
        return nullptr;
    }
    if (n0 > 1024) {
        why = "species 0 extent above 1024";
        return nullptr;
    }
    std::unique_ptr<PlaneData> pd(new PlaneData());
    const int nr = m.nr, ns = m.ns;
    const bool rows = ns == 3;
    pd->n0 = n0;
    pd->n1 = rows ? m.bounds[1] + 1 : 1;
    pd->n2 = m.bounds[ns - 1] + 1;
    pd->nr = nr;
    pd->tab_stride = m.tab_stride;
    std::vector<int> nu0(nr), nu1(nr), nu2(nr);
    for (int r = 0; r < nr; ++r) {
        nu0[r] = m.nu[(size_t)r * ns + 0];
        nu1[r] = rows ? m.nu[(size_t)r * ns + 1] : 0;
        nu2[r] = m.nu[(size_t)r * ns + ns - 1];
    }
    // species-0 factor slots: shifted Fa_r(x0) = f0_r(x0 - nu0) (0 outside) and unshifted Fb_r(x0)
    std::vector<std::vector<double>> fa_tabs, fb_tabs;
    std::vector<int> fa_slot(nr), fb_slot(nr), fa_rep, fb_rep;
    for (int r = 0; r < nr; ++r) {
        const double *t = m.tables.data() + (size_t)r * m.tab_stride;
        std::vector<double> a(n0), b(t, t + n0);
        for (int x = 0; x < n0; ++x) {
            const int xs = x - nu0[r];
            a[x] = (xs < 0 || xs >= n0) ? 0.0 : t[xs];
        }
        fa_slot[r] = all_ones(a) ? -1 : intern(fa_tabs, a);
        if (fa_slot[r] >= (int)fa_rep.size()) fa_rep.push_back(r);
        fb_slot[r] = all_ones(b) ? -1 : intern(fb_tabs, b);
        if (fb_slot[r] >= (int)fb_rep.size()) fb_rep.push_back(r);
    }
    // distinct offsets, shifted terms (offset, Fa slot), diagonal groups (Fb slot)
    std::vector<std::vector<int>> offs;
    std::vector<std::pair<int, int>> terms;
    std::vector<int> dgs;
    std::vector<int> r_term(nr), r_dg(nr), o0, o1, o2, t_off, t_fa, dg_fb;
    for (int r = 0; r < nr; ++r) {
        const int k = intern(offs, std::vector<int>{nu0[r], nu1[r], nu2[r]});
        r_term[r] = intern(terms, std::make_pair(k, fa_slot[r]));
        r_dg[r] = intern(dgs, fb_slot[r]);
    }
    for (auto &o : offs) {
        o0.push_back(o[0]);
        o1.push_back(o[1]);
        o2.push_back(o[2]);
    }
    for (auto &t : terms) {
        t_off.push_back(t.first);
        t_fa.push_back(t.second);
    }
    dg_fb = dgs;
    std::memset(&pd->wa, 0, sizeof(pd->wa));
    pd->wa.nr = nr;
    pd->wa.nt = (int)terms.size();
    pd->wa.nw = (int)(terms.size() + dgs.size());
    pd->wa.nwp = (pd->wa.nw + 1) & ~1;
    for (int r = 0; r < nr; ++r) {
        pd->wa.r_term[r] = r_term[r];
        pd->wa.r_dg[r] = r_dg[r];
    }
    // Tile rows TR (dividing n1; 2 unless CUFSP_PLANE_TR says otherwise, stepping down when nothing
    // fits) and ring stages S (3..5, or exactly CUFSP_PLANE_STAGES when set).  Occupancy comes first:
    // among the stage counts that fit, take the one giving the most CTAs per SM -- bounded by the
    // ring's shared memory and by 128 registers per thread -- and the most stages among those.
    // (At 255^3: S = 4 with 4 CTAs/SM moves 5.2 TB/s where S = 5 with 3 CTAs/SM moves 4.85.)
    const int chunks = (n0 + 63) / 64;
    pd->threads = 32 * chunks;
    pd->pitch = 64 * chunks;
    const int ytma = env_int("CUFSP_PLANE_YTMA", 1) != 0 ? 1 : 0;
    const int pps = env_int("CUFSP_PLANE_PPS", 1) == 2 ? 2 : 1;  // planes per CTA barrier
    const DeviceInfo &di = device_info();
    const int want_tr = env_int("CUFSP_PLANE_TR", 2);
    const int env_s = env_int("CUFSP_PLANE_STAGES", 0);
    const int min_s = pps == 2 ? 4 : 3;
    const int max_s = env_s > 0 ? std::max(min_s, std::min(12, env_s)) : 5;
    auto stage_bytes = [&](int tr_, bool accum) {
        const int nq_ = rows ? tr_ + 2 : 1;
        return (size_t)8 * ((size_t)(nq_ + (accum && ytma ? tr_ : 0)) * pd->pitch + (size_t)tr_ * pd->wa.nwp);
    };
    const int by_regs = std::max(1, 65536 / (128 * pd->threads));
    auto ctas_per_sm = [&](size_t smem) {
        return std::min(by_regs, (int)std::max<size_t>(1, (size_t)(di.max_smem_optin + 1024) / (smem + 1024)));
    };
    int tr = 0, stages = 0;
    for (int cand : {want_tr, 4, 2, 1}) {
        if (tr) break;
        if (cand < 1 || cand > 8 || (rows ? pd->n1 % cand != 0 : cand != 1)) continue;
        if (cand > want_tr && want_tr >= 1) continue;
        int best_occ = 0;
        for (int st = max_s; st >= (env_s > 0 ? max_s : min_s); --st) {
            const size_t b = st * stage_bytes(cand, true);
            if (b > (size_t)di.max_smem_optin) continue;
            const int occ = ctas_per_sm(b);
            if (occ > best_occ) {
                best_occ = occ;
                tr = cand;
                stages = st;
            }
        }
        if (!tr && env_s > 0)  // the requested stage count does not fit: step down as far as needed
            for (int st = max_s - 1; st >= min_s && !tr; --st)
                if (st * stage_bytes(cand, true) <= (size_t)di.max_smem_optin) {
                    tr = cand;
                    stages = st;
                }
    }
    if (!tr) {
        why = "ring stages exceed shared memory";
        return nullptr;
    }
    pd->tr = tr;
    pd->row_blocks = pd->n1 / tr;
    pd->smem_accum = stages * stage_bytes(tr, true);
    pd->smem_set = stages * stage_bytes(tr, false);
    // CTAs per SM the launch bounds promise (the occupancy the shape was chosen for).
    const int minb = std::max(1, std::min(16, env_int("CUFSP_PLANE_MINB", ctas_per_sm(pd->smem_accum))));
    std::ostringstream s;
    s << "#define CUFSP_PLANE_NR " << nr << "\n#define CUFSP_PLANE_NOFF " << offs.size() << "\n#define CUFSP_PLANE_NFA "
      << fa_tabs.size() << "\n#define CUFSP_PLANE_NFB " << fb_tabs.size() << "\n#define CUFSP_PLANE_NT " << terms.size()
      << "\n#define CUFSP_PLANE_NDG " << dgs.size() << "\n#define CUFSP_PLANE_TR " << tr << "\n#define CUFSP_PLANE_STAGES "
      << stages << "\n#define CUFSP_PLANE_PPS " << pps << "\n#define CUFSP_PLANE_YTMA " << ytma << "\n#define CUFSP_PLANE_ROWS " << (rows ? 1 : 0) << "\n#define CUFSP_PLANE_THREADS " << pd->threads
      << "\n#define CUFSP_PLANE_MINB " << minb << "\n";
    // Tries of the bounded waits before a plane is computed (tests of the watchdog only).
    if (const char *wt = getenv("CUFSP_PLANE_WAIT_TRIES")) s << "#define CUFSP_PLANE_WAIT_TRIES " << std::max(0, atoi(wt)) << "\n";
    s << "namespace cufsp_plane {\n";
    emit_fn(s, "nu0", nu0);
    emit_fn(s, "o0", o0);
    emit_fn(s, "o1", o1);
    emit_fn(s, "o2", o2);
    emit_fn(s, "t_off", t_off);
    emit_fn(s, "t_fa", t_fa);
    emit_fn(s, "r_term", r_term);
    emit_fn(s, "r_dg", r_dg);
    emit_fn(s, "fa_rep", fa_rep);
    emit_fn(s, "fb_rep", fb_rep);
    emit_fn(s, "dg_fb", dg_fb);
    s << "}\n";
    const std::string src = s.str() + kPlaneSource;
    pd->k = rtc_module(src, {"cufsp_plane_mv_accum", "cufsp_plane_mv_set"}, why);
    if (!pd->k) return nullptr;
    const void *k_accum = (const void *)pd->k->kernels[0], *k_set = (const void *)pd->k->kernels[1];
    cudaError_t e = cudaFuncSetAttribute(k_accum, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pd->smem_accum);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_set, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pd->smem_set);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pd->occ_accum, k_accum, pd->threads, pd->smem_accum);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pd->occ_set, k_set, pd->threads, pd->smem_set);
    if (e != cudaSuccess || pd->occ_accum < 1 || pd->occ_set < 1) {
        cudaGetLastError();
        why = "plane kernel does not fit an SM";
        return nullptr;
    }

    // outer factors G[q][r] for q = x1 + n1 * x2 (all species but 0)
    const int64_t Q = (int64_t)pd->n1 * pd->n2;
    std::vector<double2> g((size_t)Q * nr);
    for (int64_t q = 0; q < Q; ++q) {
        const int xs1 = rows ? (int)(q % pd->n1) : 0;
        const int xs2 = (int)(q / pd->n1);
        for (int r = 0; r < nr; ++r) {
            const double *tr_ = m.tables.data() + (size_t)r * m.tab_stride;
            double ga = 1.0, gb = 1.0;
            bool ok = true;
            for (int sp = 1; sp < ns; ++sp) {
                const int xs = sp == ns - 1 ? xs2 : xs1;
                const double *t = tr_ + m.tab_off[sp];
                gb *= t[xs];
                const int xsh = xs - m.nu[(size_t)r * ns + sp];
                if (xsh < 0 || xsh > m.bounds[sp]) ok = false;
                else ga *= t[xsh];
            }
            g[(size_t)q * nr + r] = make_double2(ok ? ga : 0.0, gb);
        }
    }
    e = dev_malloc(&pd->d_gtab, sizeof(double2) * g.size());
    if (e == cudaSuccess) e = cudaMemcpy(pd->d_gtab, g.data(), sizeof(double2) * g.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = upload_fence();
    if (e == cudaSuccess && !(pd->h_err = watch_word_alloc(&pd->d_err))) e = cudaErrorMemoryAllocation;
    if (e == cudaSuccess) e = dev_malloc(&pd->d_words, sizeof(double) * (size_t)Q * pd->wa.nwp);
    if (e != cudaSuccess) {
        cudaGetLastError();
        why = std::string("plane kernel tables: ") + cudaGetErrorString(e);
        plane_destroy(pd.release());
        return nullptr;
    }
    pd->d_tab0 = d_tables;  // species 0 is the first block of every reaction's tables
    std::ostringstream d;
    d << "plane kernel (NVRTC, sm_100a, TMA ring): NR=" << nr << " offsets=" << offs.size() << " terms=" << terms.size()
      << " diag groups=" << dgs.size() << " factor slots=" << fa_tabs.size() << "+" << fb_tabs.size() << " TR=" << tr
      << " stages=" << stages << " planes/step=" << pps << " ytma=" << ytma << " threads=" << pd->threads << " CTAs/SM=" << pd->occ_accum;
    pd->description = d.str();
    return pd.release();
}

void plane_destroy(PlaneData *pd) {
    if (!pd) return;
    if (pd->d_gtab) cudaFree(pd->d_gtab);
    watch_word_free(pd->h_err);
    if (pd->d_words) cudaFree(pd->d_words);
    delete pd;  // the compiled kernels stay in the process cache
}

const std::string &plane_description(const PlaneData *pd) { return pd->description; }
int64_t plane_size(const PlaneData *pd) { return (int64_t)pd->n0 * pd->n1; }

int plane_watchdog(PlaneData *pd) { return watch_word_take(pd->h_err); }

// Row words for these coefficients, rebuilt in stream order when they change.
cufsp_status plane_prepare(PlaneData *pd, const double *coefs, cudaStream_t st) {
    std::vector<double> cv(coefs, coefs + pd->nr);
    if (cv == pd->words_coefs) return CUFSP_SUCCESS;
    for (int r = 0; r < pd->nr; ++r) pd->wa.coef[r] = cv[r];
    const int64_t rows = (int64_t)pd->n1 * pd->n2;
    const int64_t tot = rows * pd->wa.nwp;
    k_plane_words<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(pd->wa, pd->d_gtab, rows, pd->d_words);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        pd->words_coefs.clear();
        return cuda_error(e, "plane row words");
    }
    pd->words_coefs = cv;
    return CUFSP_SUCCESS;
}

bool plane_launch(PlaneData *pd, const double *coefs, double alpha, const double *d_alpha, const int *d_skip,
                  const double *x, bool accumulate, double *y, cudaStream_t st, int64_t i_begin, int64_t i_end,
                  cufsp_status *status) {
    const int64_t P = (int64_t)pd->n0 * pd->n1;
    const int64_t n = P * pd->n2;
    if (i_end < 0) i_end = n;
    if (i_begin % P != 0 || i_end % P != 0) return false;
    if (((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % 16) != 0) return false;
    *status = CUFSP_SUCCESS;
    const int zb = (int)(i_begin / P), ze = (int)(i_end / P);
    if (ze <= zb) return true;
    {
        const cufsp_status ws = plane_prepare(pd, coefs, st);
        if (ws != CUFSP_SUCCESS) {
            *status = ws;
            return true;
        }
    }
    CufspPlaneArgs a;
    std::memset(&a, 0, sizeof(a));
    a.words = pd->d_words;
    a.tab0 = pd->d_tab0;
    a.d_alpha = d_alpha;
    a.d_skip = d_skip;
    a.err = pd->d_err;
    a.n0 = pd->n0;
    a.n1 = pd->n1;
    a.n2 = pd->n2;
    a.tab_stride = pd->tab_stride;
    a.pitch = pd->pitch;
    a.row_blocks = pd->row_blocks;
    a.z_begin = zb;
    a.z_end = ze;
    a.alpha = alpha;
    a.nwp = pd->wa.nwp;
    // Plane segments: fill the resident CTA slots in as few waves as possible, counting the two
    // extra planes every segment reads around its output planes.
    const int planes = ze - zb;
    const int64_t slots = (int64_t)device_info().sm_count * (accumulate ? pd->occ_accum : pd->occ_set);
    int nseg = env_int("CUFSP_PLANE_NSEG", 0);
    if (nseg <= 0) {
        double best = 1e300;
        for (int sgs = 1; sgs <= planes; ++sgs) {
            const int zs = (planes + sgs - 1) / sgs;
            const int real = (planes + zs - 1) / zs;
            const int64_t items = (int64_t)pd->row_blocks * real;
            const double waves = (double)((items + slots - 1) / slots);
            const double cost = waves * (zs + 2);
            if (cost < best - 1e-9) {
                best = cost;
                nseg = real;
            }
            if (items > 8 * slots) break;
        }
    }
    nseg = std::max(1, std::min(nseg, planes));
    a.zseg = (planes + nseg - 1) / nseg;
    const int segs = (planes + a.zseg - 1) / a.zseg;
    a.items = pd->row_blocks * segs;
    void *args[] = {&a, (void *)&x, (void *)&y};
    cudaError_t e = cudaLaunchKernel((const void *)pd->k->kernels[accumulate ? 0 : 1], dim3((unsigned)a.items),
                                     dim3((unsigned)pd->threads), args, accumulate ? pd->smem_accum : pd->smem_set, st);
    if (e != cudaSuccess) *status = cuda_error(e, "plane kernel launch");
    return true;
}

}  // namespace cufsp
