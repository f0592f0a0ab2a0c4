// cufsp_arnoldi.cu -- the Arnoldi pass of one Krylov step as ONE persistent launch, for generators
// whose Krylov basis stays in L2 (single-instance solves of 32K-1M states).
//
// Same arithmetic contract as the launch sequence of cufsp_krylov.cu (src/KryExpvFSP.cu:38-120,
// restated there): basis W_k with v_k = rho_k W_k, h = V^T w, w -= V h, ||w||, happy breakdown,
// ||A v_m||, results in the same device state block.  At these sizes every one of the ~3m kernels
// of that sequence is latency-bound (a few microseconds of launch and grid-reduction tail each for
// well under a microsecond of L2 traffic); here one cooperative grid walks all m iterations:
//  * the generator is applied from a per-state term table built once per coefficient vector:
//      (A x)[i] = sum_t coef[t][i] x[i - shift_t]   (last term: shift 0, the diagonal),
//    coefficient 0 wherever the source state leaves the box (its index is clamped to [0, n)), so
//    the gather needs no multi-index decode; the same form holds for A^T (adjoint solves);
//  * the dot products h = V^T w are taken in the same pass that produces w = rho_j A W_j (each
//    thread owns its states for the whole launch, so its w values need no barrier);
//  * two grid barriers per iteration (after the dots, after the norm); each barrier completes a
//    deterministic reduction: every CTA writes its partial sums, and after the barrier EVERY CTA
//    sums all partials in the same fixed order, so all CTAs take identical decisions;
//  * barrier waits are bounded (~0.3 s); on expiry the kernel sets an error word, every CTA leaves
//    at its next barrier, and the host reports CUFSP_ERR_CUDA.  The launch is cooperative, so all
//    CTAs are co-resident.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>

#include <mutex>

#include "cufsp_internal.h"

namespace cufsp {

namespace {

constexpr int kPThreads = 1024;
constexpr int kPWarps = kPThreads / 32;
constexpr int kKMax = 64;            // partial sums per CTA (>= CUFSP_MAX_KRYLOV)
constexpr int kMaxTerms = 64;
constexpr unsigned long long kWaitNs = 300ull * 1000 * 1000;  // a grid barrier gives up after 0.3 s

struct PArgs {
    int64_t n;
    int64_t chunk;              // states per CTA (the last CTA may have fewer)
    int T;
    const double *coef;         // [T][n]
    int64_t shift[kMaxTerms];   // source index i - shift[t] (clamped)
    const double *v0;           // W_0 (the caller's vector)
    double *W;                  // W_1 .. W_{m+1}
    double *H, *rho, *gam, *beta, *avnorm;
    int *flag;                  // 0 ok, >0 happy breakdown at mb = flag, -1 NaN/Inf, -2 zero vector
    int mp2, m, iop, q;
    double btol;
    int with_avnorm;
    double *part;               // [2][kKMax][gridDim.x] (k-major)
    unsigned *bar;              // arrival counter, zero at launch
    int *err;                   // set when a barrier wait expired
};

struct PSmem {
    double wsum[kPWarps];
    double res[kKMax];
    double rho[CUFSP_MAX_KRYLOV + 2];
    double gam[kKMax];
    int ok;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid barrier number `epoch` (1, 2, ...): the arrival counter reaches epoch * gridDim.x.
__device__ __forceinline__ bool grid_sync(const PArgs &a, unsigned &epoch, int &ok_s) {
    __syncthreads();
    ++epoch;
    if (threadIdx.x == 0) {
        // arrival with release semantics (the CTA's partial sums and w become visible first), then a
        // tight acquire poll; a measured cooperative probe: 1.26 us per barrier over 148 CTAs, against
        // 1.39-1.64 us for a fence, a relaxed atomic and 64 ns sleeps between polls.  The wait is
        // bounded by the global timer (kWaitNs); the error word is looked at every 64 polls.
        asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(a.bar), "r"(1u) : "memory");
        const unsigned target = epoch * gridDim.x;
        int ok = 1;
        const unsigned long long t0 = global_ns();
        for (int it = 1; ld_acquire(a.bar) < target; ++it) {
            if ((it & 63) == 0) {
                if (*(volatile int *)a.err) {  // another CTA gave up
                    ok = 0;
                    break;
                }
                if (global_ns() - t0 > kWaitNs) {
                    atomicExch(a.err, 1);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        ok_s = ok && *(volatile int *)a.err == 0;
    }
    __syncthreads();
    return ok_s != 0;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Grid totals of the K per-CTA partials already stored in part[0..K)[blockIdx.x] (k-major) into
// sm.res, identical in every CTA: all threads copy the K x G partials into shared memory in one
// coalesced pass, then one warp per k sums them in a fixed order.  False when a barrier wait expired.
__device__ __forceinline__ bool finish_reduce(int K, const double *part, double *red, PSmem &sm, const PArgs &a,
                                              unsigned &epoch) {
    if (!grid_sync(a, epoch, sm.ok)) return false;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int G = gridDim.x;
    for (int p = threadIdx.x; p < K * G; p += blockDim.x) red[p] = __ldcg(part + p);
    __syncthreads();
    for (int k = warp; k < K; k += kPWarps) {
        double v = 0.0;
        for (int b = lane; b < G; b += 32) v += red[k * G + b];
        v = warp_sum(v);
        if (lane == 0) sm.res[k] = v;
    }
    __syncthreads();
    return true;
}

// Block sum of one value per thread into part[0][blockIdx.x] (fixed order), then finish_reduce.
__device__ __forceinline__ bool reduce1(double v, double *part, double *red, PSmem &sm, const PArgs &a,
                                        unsigned &epoch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) sm.wsum[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double t = warp_sum(sm.wsum[lane]);
        if (lane == 0) __stcg(part + blockIdx.x, t);
    }
    return finish_reduce(1, part, red, sm, a, epoch);
}

// (A x)[i] from the term table (one state).
__device__ __forceinline__ double term_apply(const PArgs &a, const double *x, int64_t i) {
    double s = 0.0;
    for (int t = 0; t < a.T; ++t) {
        int64_t src = i - a.shift[t];
        src = src < 0 ? 0 : (src >= a.n ? a.n - 1 : src);
        s = fma(__ldg(a.coef + (size_t)t * a.n + i), __ldcg(x + src), s);
    }
    return s;
}

// CTA b owns the states [b chunk, (b + 1) chunk); its slice of the newest vector w lives in shared
// memory (ws) as well as in global memory (for the other CTAs' neighbour gathers).
__global__ void __launch_bounds__(kPThreads, 1) k_arnoldi_persistent(const PArgs a) {
    extern __shared__ double ws[];  // [chunk] own slice of w, then [m][gridDim.x] partial sums
    __shared__ PSmem sm;
    const int64_t n = a.n;
    const int64_t lo = (int64_t)blockIdx.x * a.chunk;
    const int len = (int)max((int64_t)0, min(a.chunk, n - lo));
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool lead = blockIdx.x == 0 && tid == 0;
    const int mp2 = a.mp2;
    unsigned epoch = 0;
    int rc = 0;
    auto part = [&]() { return a.part + (size_t)((rc++) & 1) * gridDim.x * kKMax; };
    auto wv = [&](int k) -> const double * { return k == 0 ? a.v0 : a.W + (size_t)(k - 1) * n; };
    double *red = ws + a.chunk;

    if (blockIdx.x == 0) {
        for (int i = tid; i < mp2 * mp2; i += blockDim.x) a.H[i] = 0.0;
        for (int i = tid; i < mp2; i += blockDim.x) {
            a.rho[i] = 0.0;
            a.gam[i] = 0.0;
        }
    }
    double acc = 0.0;
    for (int il = tid; il < len; il += blockDim.x) {
        const double t = __ldcg(a.v0 + lo + il);
        acc = fma(t, t, acc);
    }
    if (!reduce1(acc, part(), red, sm, a, epoch)) return;
    const double beta = sqrt(sm.res[0]);
    const int flag0 = !isfinite(beta) ? -1 : (beta == 0.0 ? -2 : 0);
    if (tid == 0) sm.rho[0] = beta > 0.0 ? 1.0 / beta : 0.0;
    __syncthreads();  // block 0's clearing of rho/gam precedes the writes below
    if (lead) {
        *a.beta = beta;
        *a.avnorm = 0.0;
        a.rho[0] = sm.rho[0];
        *a.flag = flag0;
    }
    if (flag0) return;

    for (int j = 0; j < a.m; ++j) {
        const int istart = a.iop ? max(0, j - a.q + 1) : 0;
        const int K = j - istart + 1;
        const double *x = wv(j);
        double *w = a.W + (size_t)j * n;  // W_{j+1}
        const double rj = sm.rho[j];
        // w = rho_j A W_j on the own slice
        for (int il = tid; il < len; il += blockDim.x) {
            const double wi = rj * term_apply(a, x, lo + il);
            ws[il] = wi;
            __stcg(w + lo + il, wi);
        }
        __syncthreads();
        // h_k partials: one warp per basis vector, w from shared memory
        {
            double *pp = part();
            for (int k = warp; k < K; k += kPWarps) {
                const double *vk = wv(istart + k) + lo;
                double d = 0.0;
                for (int il = lane; il < len; il += 32) d = fma(__ldcg(vk + il), ws[il], d);
                d = warp_sum(d);
                if (lane == 0) __stcg(pp + (size_t)k * gridDim.x + blockIdx.x, d);
            }
            if (!finish_reduce(K, pp, red, sm, a, epoch)) return;
        }
        if (tid < K) {
            const int kk = istart + tid;
            const double r = sm.rho[kk];
            const double h = r * sm.res[tid];
            sm.gam[tid] = h * r;
            if (blockIdx.x == 0) {
                a.H[kk + (size_t)j * mp2] = h;
                a.gam[kk] = h * r;
            }
        }
        __syncthreads();
        // w -= sum_k gam_k W_k and ||w||^2
        acc = 0.0;
        for (int il = tid; il < len; il += blockDim.x) {
            double wi = ws[il];
            for (int k = 0; k < K; ++k) wi = fma(-sm.gam[k], __ldcg(wv(istart + k) + lo + il), wi);
            __stcg(w + lo + il, wi);
            acc = fma(wi, wi, acc);
        }
        if (!reduce1(acc, part(), red, sm, a, epoch)) return;
        const double sn = sqrt(sm.res[0]);
        if (!isfinite(sn)) {
            if (lead) *a.flag = -1;
            return;
        }
        if (sn < a.btol) {
            if (lead) *a.flag = j + 1;
            return;
        }
        if (tid == 0) sm.rho[j + 1] = 1.0 / sn;
        if (lead) {
            a.H[(j + 1) + (size_t)j * mp2] = sn;
            a.rho[j + 1] = 1.0 / sn;
        }
        __syncthreads();
    }
    if (a.with_avnorm) {  // ||A v_m|| (src/KryExpvFSP.cu:114-120)
        const double *x = wv(a.m);
        double *w = a.W + (size_t)a.m * n;
        const double rm = sm.rho[a.m];
        acc = 0.0;
        for (int il = tid; il < len; il += blockDim.x) {
            const double wi = rm * term_apply(a, x, lo + il);
            __stcg(w + lo + il, wi);
            acc = fma(wi, wi, acc);
        }
        if (!reduce1(acc, part(), red, sm, a, epoch)) return;
        if (lead) {
            const double av = sqrt(sm.res[0]);
            *a.avnorm = av;
            if (!isfinite(av)) *a.flag = -1;
        }
    }
}

// ---- term table ---------------------------------------------------------------------------------

struct TermBuildArgs {
    int64_t n;
    int ns, nr, T, tab_stride, transpose;
    int dims[CUFSP_MAX_SPECIES];
    int tab_off[CUFSP_MAX_SPECIES];
    const double *tables;  // [nr][tab_stride] factor tables, or null
    const double *props;   // [nr][n] propensities a_r(x_i), or null
    const int *nu;         // [nr][ns]
    const double *c;       // [nr] coefficients
    const int *rterm;      // [nr] term of reaction r (-1: no net change)
    const int64_t *d;      // [nr] flat shift sum_s nu_{r,s} stride_s
    double *coef;          // [T][n]
};

__device__ __forceinline__ double prop_at(const TermBuildArgs &b, int r, int64_t i, const int *xs) {
    if (b.props) return b.props[(size_t)r * b.n + i];
    double f = 1.0;
    const double *tr = b.tables + (size_t)r * b.tab_stride;
    for (int s = 0; s < b.ns; ++s) f *= tr[b.tab_off[s] + xs[s]];
    return f;
}

__global__ void k_build_terms(const TermBuildArgs b) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b.n; i += stride) {
        int xs[CUFSP_MAX_SPECIES], ys[CUFSP_MAX_SPECIES];
        int64_t rem = i;
        for (int s = 0; s < b.ns; ++s) {
            xs[s] = (int)(rem % b.dims[s]);
            rem /= b.dims[s];
        }
        double acc[kMaxTerms];
        for (int t = 0; t < b.T; ++t) acc[t] = 0.0;
        for (int r = 0; r < b.nr; ++r) {
            const double cr = b.c[r];
            const double here = prop_at(b, r, i, xs);
            acc[b.T - 1] -= cr * here;  // the diagonal keeps the full outflow
            const int t = b.rterm[r];
            if (t < 0) continue;
            const int sg = b.transpose ? 1 : -1;  // A: source x - nu_r;  A^T: target x + nu_r
            bool ok = true;
            for (int s = 0; s < b.ns; ++s) {
                ys[s] = xs[s] + sg * b.nu[r * b.ns + s];
                ok = ok && ys[s] >= 0 && ys[s] < b.dims[s];
            }
            if (!ok) continue;
            if (b.transpose) acc[t] += cr * here;
            else acc[t] += cr * prop_at(b, r, i - b.d[r], ys);
        }
        for (int t = 0; t < b.T; ++t) b.coef[(size_t)t * b.n + i] = acc[t];
    }
}

thread_local bool tl_disabled = false;

}  // namespace

struct PArnoldi {
    struct Terms {
        std::vector<double> coefs;
        bool transpose = false;
        int T = 0;
        std::vector<int64_t> shift;
        double *d_coef = nullptr;
    };
    Terms terms[2];       // forward and transposed, each for its last coefficient vector
    int *d_nu = nullptr;  // model data for the term builder
    double *d_tables = nullptr, *d_c = nullptr;
    int *d_rterm = nullptr;
    int64_t *d_d = nullptr;
    double *d_props = nullptr;  // sparse formats: exported propensities
    double *d_part = nullptr;
    unsigned *d_bar = nullptr;  // grid-barrier arrival counter
    int grid = 0;
    int64_t chunk = 0;
    size_t smem = 0;
};

namespace {
template <class Free>
void parnoldi_release(PArnoldi *pa, Free release) {
    if (!pa) return;
    for (auto &t : pa->terms) release(t.d_coef);
    release(pa->d_nu);
    release(pa->d_tables);
    release(pa->d_c);
    release(pa->d_rterm);
    release(pa->d_d);
    release(pa->d_props);
    release(pa->d_part);
    release(pa->d_bar);
    delete pa;
}
}  // namespace

void parnoldi_destroy(PArnoldi *pa) {
    parnoldi_release(pa, [](void *p) { cache_free(p); });
}

void parnoldi_destroy(PArnoldi *pa, cudaStream_t last_use) {
    parnoldi_release(pa, [last_use](void *p) { cache_free(p, last_use); });
}

void parnoldi_thread_disable(bool off) { tl_disabled = off; }

namespace {
thread_local int tl_cta_cap = 0;  // at most this many CTAs per pass launched from this thread (0: all SMs)
}
void parnoldi_thread_cta_cap(int cap) { tl_cta_cap = cap > 0 ? cap : 0; }

namespace {
int persistent_mode() {  // CUFSP_ARNOLDI_PERSISTENT: 0 never, 1 always, unset: by size
    static const int mode = [] {
        const char *e = getenv("CUFSP_ARNOLDI_PERSISTENT");
        return e ? atoi(e) : -1;
    }();
    return mode;
}
}  // namespace

bool parnoldi_size_ok(int64_t n) {
    static const int64_t max_n = [] {
        const char *e = getenv("CUFSP_ARNOLDI_MAX_N");
        return e ? (int64_t)atoll(e) : (int64_t)1 << 20;
    }();
    const int mode = persistent_mode();
    return mode != 0 && (mode == 1 || n <= max_n);
}

bool parnoldi_wanted(const cufsp_mat *A, int64_t n, int m) {
    if (tl_disabled || !A || m > CUFSP_MAX_KRYLOV || !parnoldi_size_ok(n)) return false;
    if (A->model.nr > CUFSP_MAX_REACTIONS_SPARSE || A->model.ns > CUFSP_MAX_SPECIES) return false;
    return A->format == CUFSP_FORMAT_KRONECKER ? !A->model.tables.empty() : A->sparse != nullptr;
}

namespace {

// Term table of A (or A^T) at `coefs`, rebuilt when either changes.
cufsp_status build_terms(PArnoldi *pa, cufsp_mat *A, const std::vector<double> &coefs, bool transpose,
                         PArnoldi::Terms *&out, cudaStream_t st) {
    PArnoldi::Terms &tm = pa->terms[transpose ? 1 : 0];
    out = &tm;
    if (tm.d_coef && tm.transpose == transpose && tm.coefs == coefs) return CUFSP_SUCCESS;
    const ModelHost &m = A->model;
    const int ns = m.ns, nr = m.nr;
    const int64_t n = m.n;
    // flat shifts and their distinct values (shift 0 = no net change)
    std::vector<int64_t> d(nr, 0), stride(ns, 1);
    for (int s = 1; s < ns; ++s) stride[s] = stride[s - 1] * ((int64_t)m.bounds[s - 1] + 1);
    for (int r = 0; r < nr; ++r)
        for (int s = 0; s < ns; ++s) d[r] += (int64_t)m.nu[(size_t)r * ns + s] * stride[s];
    std::map<int64_t, int> idx;
    std::vector<int> rterm(nr, -1);
    std::vector<int64_t> shifts;
    for (int r = 0; r < nr; ++r) {
        if (d[r] == 0) continue;
        const int64_t sh = transpose ? -d[r] : d[r];
        auto it = idx.find(sh);
        if (it == idx.end()) {
            it = idx.emplace(sh, (int)shifts.size()).first;
            shifts.push_back(sh);
        }
        rterm[r] = it->second;
    }
    const int T = (int)shifts.size() + 1;
    if (T > kMaxTerms) return set_error(CUFSP_ERR_UNSUPPORTED, "persistent Arnoldi: more than 63 distinct shifts");
    shifts.push_back(0);
    // model data on the device (once per generator), in order on st like the build below
    if (!pa->d_nu) {
        CUFSP_CUDA_TRY(cache_alloc((void **)&pa->d_nu, sizeof(int) * (size_t)nr * ns));
        CUFSP_CUDA_TRY(cudaMemcpyAsync(pa->d_nu, m.nu.data(), sizeof(int) * (size_t)nr * ns, cudaMemcpyHostToDevice, st));
        CUFSP_CUDA_TRY(cache_alloc((void **)&pa->d_c, sizeof(double) * nr));
        CUFSP_CUDA_TRY(cache_alloc((void **)&pa->d_rterm, sizeof(int) * nr * 2));
        CUFSP_CUDA_TRY(cache_alloc((void **)&pa->d_d, sizeof(int64_t) * nr));
        CUFSP_CUDA_TRY(cudaMemcpyAsync(pa->d_d, d.data(), sizeof(int64_t) * nr, cudaMemcpyHostToDevice, st));
        if (A->format == CUFSP_FORMAT_KRONECKER) {
            CUFSP_CUDA_TRY(cache_alloc((void **)&pa->d_tables, sizeof(double) * m.tables.size()));
            CUFSP_CUDA_TRY(cudaMemcpyAsync(pa->d_tables, m.tables.data(), sizeof(double) * m.tables.size(),
                                           cudaMemcpyHostToDevice, st));
        }
    }
    TermBuildArgs b;
    std::memset(&b, 0, sizeof(b));
    b.n = n;
    b.ns = ns;
    b.nr = nr;
    b.T = T;
    b.transpose = transpose ? 1 : 0;
    b.tab_stride = m.tab_stride;
    for (int s = 0; s < ns; ++s) {
        b.dims[s] = m.bounds[s] + 1;
        b.tab_off[s] = m.tab_off.empty() ? 0 : m.tab_off[s];
    }
    if (A->format == CUFSP_FORMAT_KRONECKER) {
        b.tables = pa->d_tables;
    } else {
        if (!pa->d_props) CUFSP_CUDA_TRY(cache_alloc((void **)&pa->d_props, sizeof(double) * (size_t)nr * n));
        cufsp_status s = sparse_export(A->sparse, pa->d_props, st);
        if (s != CUFSP_SUCCESS) return s;
        b.props = pa->d_props;
    }
    // per-call coefficients and term map: small copies in stream order
    int *d_rt = pa->d_rterm + (transpose ? nr : 0);
    CUFSP_CUDA_TRY(cudaMemcpyAsync(pa->d_c, coefs.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, st));
    CUFSP_CUDA_TRY(cudaMemcpyAsync(d_rt, rterm.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, st));
    b.nu = pa->d_nu;
    b.c = pa->d_c;
    b.rterm = d_rt;
    b.d = pa->d_d;
    if (!tm.d_coef || tm.T < T) {
        cache_free(tm.d_coef);
        tm.d_coef = nullptr;
        CUFSP_CUDA_TRY(cache_alloc((void **)&tm.d_coef, sizeof(double) * (size_t)T * n));
    }
    b.coef = tm.d_coef;
    const int grid = stream_grid(n, 1, device_info().sm_count * 8);
    k_build_terms<<<grid, 256, 0, st>>>(b);
    CUFSP_CUDA_TRY(cudaGetLastError());
    // the copies above read pageable host memory: finish before `rterm` goes out of scope
    CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
    tm.coefs = coefs;
    tm.transpose = transpose;
    tm.T = T;
    tm.shift = shifts;
    return CUFSP_SUCCESS;
}

}  // namespace

namespace {
cudaError_t persistent_smem_attribute() {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static bool done[kMaxDevices] = {};
    static cudaError_t result[kMaxDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(mu);
    if (!done[dev]) {
        result[dev] = cudaFuncSetAttribute((const void *)k_arnoldi_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           device_info().max_smem_optin - (int)sizeof(PSmem) - 1024);
        done[dev] = true;
    }
    return result[dev];
}
}  // namespace

cufsp_status parnoldi_run(PArnoldi **ppa, cufsp_mat *A, const std::vector<double> &coefs, bool transpose,
                          int64_t n, const double *v, double *W, double *H, double *rho, double *gam, double *beta,
                          double *avnorm, int *flag, int *err, int m, int iop, int q, double btol, bool with_avnorm,
                          cudaStream_t st) {
    if (!*ppa) *ppa = new PArnoldi();
    PArnoldi *pa = *ppa;
    PArnoldi::Terms *tm = nullptr;
    cufsp_status s = build_terms(pa, A, coefs, transpose, tm, st);
    if (s != CUFSP_SUCCESS) return s;
    if (!pa->grid) {
        // One CTA per SM (fewer for small n: at least 256 states each by default); the CTA's slice
        // of the newest vector must fit its shared memory.
        static const int64_t min_states = [] {  // states per CTA at least (CUFSP_ARNOLDI_CTA_STATES)
            const char *e = getenv("CUFSP_ARNOLDI_CTA_STATES");
            return e ? std::max<int64_t>(32, atoll(e)) : (int64_t)256;
        }();
        // a host thread that shares the GPU with other solves (the batched gradient's workers) takes
        // its share of the SMs, so that the workers' cooperative passes run side by side
        const int sms = tl_cta_cap > 0 ? std::min(tl_cta_cap, device_info().sm_count) : device_info().sm_count;
        const int64_t want = std::max<int64_t>(1, std::min<int64_t>(sms, (n + min_states - 1) / min_states));
        const int64_t chunk = (n + want - 1) / want;
        const int64_t grid = (n + chunk - 1) / chunk;
        const size_t smem = sizeof(double) * ((size_t)chunk + (size_t)std::max(1, m) * grid);
        if (smem > (size_t)device_info().max_smem_optin - sizeof(PSmem) - 1024)
            return set_error(CUFSP_ERR_UNSUPPORTED, "persistent Arnoldi: vector slice exceeds shared memory");
        // The attribute belongs to the current device: set it once per device, to the most any
        // driver may ask for, so that drivers of different sizes on different host threads never
        // undercut each other.
        CUFSP_CUDA_TRY(persistent_smem_attribute());
        int per_sm = 0;
        CUFSP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k_arnoldi_persistent,
                                                                     kPThreads, smem));
        if (per_sm < 1) return set_error(CUFSP_ERR_CUDA, "persistent Arnoldi: kernel does not fit an SM");
        pa->grid = (int)grid;
        pa->chunk = chunk;
        pa->smem = smem;
        CUFSP_CUDA_TRY(cache_alloc((void **)&pa->d_part, sizeof(double) * 2 * (size_t)pa->grid * kKMax));
        CUFSP_CUDA_TRY(cache_alloc((void **)&pa->d_bar, sizeof(unsigned)));
    }
    PArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = n;
    a.chunk = pa->chunk;
    a.T = tm->T;
    a.coef = tm->d_coef;
    for (int t = 0; t < tm->T; ++t) a.shift[t] = tm->shift[t];
    a.v0 = v;
    a.W = W;
    a.H = H;
    a.rho = rho;
    a.gam = gam;
    a.beta = beta;
    a.avnorm = avnorm;
    a.flag = flag;
    a.mp2 = m + 2;
    a.m = m;
    a.iop = iop;
    a.q = q;
    a.btol = btol;
    a.with_avnorm = with_avnorm ? 1 : 0;
    a.part = pa->d_part;
    a.bar = pa->d_bar;
    a.err = err;
    CUFSP_CUDA_TRY(cudaMemsetAsync(pa->d_bar, 0, sizeof(unsigned), st));
    CUFSP_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
    void *args[] = {&a};
    CUFSP_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)k_arnoldi_persistent, dim3(pa->grid), dim3(kPThreads),
                                               args, pa->smem, st));
    return CUFSP_SUCCESS;
}

}  // namespace cufsp
