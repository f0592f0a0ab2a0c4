// cufsp_common.cu -- status handling, state indexing and enumeration, model validation,
// and the basic deterministic vector reductions used by the Krylov driver.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>
#include <unordered_map>

#include "cufsp_internal.h"
#include "cufsp_reduce.cuh"

namespace cufsp {

static thread_local std::string g_last_error;

cufsp_status set_error(cufsp_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}

cufsp_status cuda_error(cudaError_t e, const char *what) {
    cudaGetLastError();  // clear a sticky-free error so later calls are not misreported
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (e == cudaErrorMemoryAllocation) return set_error(CUFSP_ERR_ALLOC, m);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return set_error(CUFSP_ERR_NO_DEVICE, m);
    return set_error(CUFSP_ERR_CUDA, m);
}

void clear_error() { g_last_error.clear(); }

// A fixed table indexed by device id: entries never move, so references handed out stay valid
// while other threads look up other devices.
const DeviceInfo &device_info() {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static DeviceInfo cache[kMaxDevices];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxDevices) dev = 0;
    std::lock_guard<std::mutex> lk(mu);
    DeviceInfo &d = cache[dev];
    if (d.sm_count == 0) {
        cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&d.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (d.sm_count <= 0) d.sm_count = 148;
    }
    return d;
}

int *watch_word_alloc(int **d_word) {
    int *h = nullptr;
    *d_word = nullptr;
    if (cudaHostAlloc((void **)&h, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    *h = 0;
    if (cudaHostGetDevicePointer((void **)d_word, h, 0) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeHost(h);
        *d_word = nullptr;
        return nullptr;
    }
    return h;
}

void watch_word_free(int *h_word) {
    if (h_word) cudaFreeHost(h_word);
}

int watch_word_take(int *h_word) {
    if (!h_word) return 0;
    volatile int *w = h_word;
    const int v = *w;
    if (v) *w = 0;
    return v;
}

FastDiv make_fastdiv(uint32_t d) {
    FastDiv f;
    f.d = d;
    uint32_t l = 0;
    while ((1ull << l) < d) ++l;
    f.shift = l;
    f.mul = (uint32_t)((((1ull << 32) * ((1ull << l) - d)) / d) + 1ull);
    return f;
}

int stream_grid(int64_t n, int elems_per_thread, int max_ctas) {
    int64_t per_cta = (int64_t)kRedThreads * elems_per_thread;
    int64_t g = (n + per_cta - 1) / per_cta;
    if (g < 1) g = 1;
    if (g > max_ctas) g = max_ctas;
    return (int)g;
}

// ---- cached device buffers -------------------------------------------------------------------
// Krylov drivers are typically created and destroyed once per solve (the reference's usage); with
// plain cudaMalloc/cudaFree every solve pays the driver's page-table work and an implicit device
// synchronisation per buffer (2-6 ms per small solve measured).  Their buffers come from this cache
// instead: a released buffer is kept and handed to the next request of a similar size on the same
// device.  Work still queued may use a released buffer, so its reuse waits for it: a release that
// names the stream all uses were ordered on records an event there, and the next owner waits for
// that event only (other streams keep running); a release without a stream synchronises the
// buffer's own device.  Idle buffers are kept up to CUFSP_CACHE_MAX_MB (default 1/32 of the device
// memory, at least 1024) per process and returned to the driver by cufsp_cache_trim() or when an
// allocation of this library fails.
namespace {
struct CachedBlock {
    void *p;
    size_t bytes;
    int dev;
    cudaEvent_t ready;  // recorded at release on the releasing stream; null after a device sync
};
struct BufferCache {
    std::mutex mu;
    std::multimap<size_t, CachedBlock> idle;  // by size
    std::unordered_map<void *, CachedBlock> live;
    size_t idle_bytes = 0;
};
BufferCache &buffer_cache() {
    static BufferCache *c = new BufferCache();  // never destroyed: no CUDA calls at process exit
    return *c;
}
size_t cache_cap() {
    static const size_t cap = [] {
        if (const char *e = getenv("CUFSP_CACHE_MAX_MB")) {
            const long long mb = atoll(e);
            return (size_t)(mb < 0 ? 0 : mb) << 20;
        }
        // default: 1/32 of the device memory, at least 1 GB (5.6 GB on a 180 GB part).  Concurrent
        // gradient workers recycle a few hundred MB each per gradient (checkpoints, bases); a cap
        // below that sends buffers back through cudaFree, which synchronises the whole device.
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            cudaGetLastError();
            total_b = 0;
        }
        return std::max<size_t>((size_t)1 << 30, total_b / 32);
    }();
    return cap;
}

// Runs f with device `dev` current and restores the caller's device.
template <class F>
void on_device(int dev, F f) {
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    f();
    if (cur != dev && cur >= 0) cudaSetDevice(cur);
}

// Frees the idle blocks of device `dev` (all devices when dev < 0); the caller holds c.mu.
size_t trim_locked(BufferCache &c, int dev) {
    size_t freed = 0;
    for (auto it = c.idle.begin(); it != c.idle.end();) {
        if (dev < 0 || it->second.dev == dev) {
            CachedBlock b = it->second;
            on_device(b.dev, [&] {
                if (b.ready) {
                    cudaEventSynchronize(b.ready);
                    cudaEventDestroy(b.ready);
                }
                cudaFree(b.p);
            });
            c.idle_bytes -= b.bytes;
            freed += b.bytes;
            it = c.idle.erase(it);
        } else {
            ++it;
        }
    }
    return freed;
}
}  // namespace

cudaError_t dev_malloc(void **p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaErrorMemoryAllocation) return e;
    cudaGetLastError();
    int dev = 0;
    cudaGetDevice(&dev);
    BufferCache &c = buffer_cache();
    {
        std::lock_guard<std::mutex> lk(c.mu);
        if (trim_locked(c, dev) == 0) return e;
    }
    return cudaMalloc(p, bytes);
}

size_t cache_trim_all() {
    BufferCache &c = buffer_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    return trim_locked(c, -1);
}

cudaError_t upload_fence() { return cudaStreamSynchronize(cudaStreamLegacy); }

namespace {
struct PinnedSlots {
    std::mutex mu;
    std::vector<double *> free;
};
PinnedSlots &pinned_slots() {
    static PinnedSlots *s = new PinnedSlots();  // never destroyed: no CUDA calls at process exit
    return *s;
}
}  // namespace

double *pinned_slot_get() {
    PinnedSlots &s = pinned_slots();
    std::lock_guard<std::mutex> lk(s.mu);
    if (s.free.empty()) {
        constexpr int kPage = 512;  // doubles per pinned page (4 KB)
        double *page = nullptr;
        if (cudaHostAlloc((void **)&page, sizeof(double) * kPage, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        for (int i = kPage - 1; i >= 0; --i) s.free.push_back(page + i);
    }
    double *p = s.free.back();
    s.free.pop_back();
    return p;
}

void pinned_slot_put(double *p) {
    if (!p) return;
    PinnedSlots &s = pinned_slots();
    std::lock_guard<std::mutex> lk(s.mu);
    s.free.push_back(p);
}

cudaError_t cache_alloc(void **p, size_t bytes) {
    *p = nullptr;
    bytes = (std::max<size_t>(bytes, 1) + 255) & ~(size_t)255;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    BufferCache &c = buffer_cache();
    {
        CachedBlock b{nullptr, 0, 0, nullptr};
        {
            std::lock_guard<std::mutex> lk(c.mu);
            for (auto it = c.idle.lower_bound(bytes); it != c.idle.end() && it->first <= 2 * bytes; ++it) {
                if (it->second.dev != dev) continue;
                b = it->second;
                c.idle.erase(it);
                c.idle_bytes -= b.bytes;
                break;
            }
        }
        if (b.p) {
            if (b.ready) {  // the previous owner's work on its stream may still use the buffer
                e = cudaEventSynchronize(b.ready);
                cudaEventDestroy(b.ready);
                b.ready = nullptr;
                if (e != cudaSuccess) return e;
            }
            std::lock_guard<std::mutex> lk(c.mu);
            c.live[b.p] = b;
            *p = b.p;
            return cudaSuccess;
        }
    }
    e = dev_malloc(p, bytes);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(c.mu);
    c.live[*p] = CachedBlock{*p, bytes, dev, nullptr};
    return cudaSuccess;
}

namespace {
void cache_release(void *p, bool have_stream, cudaStream_t st) {
    if (!p) return;
    BufferCache &c = buffer_cache();
    CachedBlock b;
    {
        std::lock_guard<std::mutex> lk(c.mu);
        auto it = c.live.find(p);
        if (it == c.live.end()) {
            cudaFree(p);
            return;
        }
        b = it->second;
        c.live.erase(it);
    }
    bool keep = true;
    on_device(b.dev, [&] {
        b.ready = nullptr;
        if (have_stream && cudaEventCreateWithFlags(&b.ready, cudaEventDisableTiming) == cudaSuccess) {
            if (cudaEventRecord(b.ready, st) != cudaSuccess) {
                cudaGetLastError();
                cudaEventDestroy(b.ready);
                b.ready = nullptr;
            }
        }
        if (!b.ready) cudaDeviceSynchronize();  // work still queued on this device may use the buffer
        std::lock_guard<std::mutex> lk(c.mu);
        if (c.idle_bytes + b.bytes > cache_cap()) {
            if (b.ready) {
                cudaEventSynchronize(b.ready);
                cudaEventDestroy(b.ready);
            }
            cudaFree(b.p);
            keep = false;
        }
    });
    if (!keep) return;
    std::lock_guard<std::mutex> lk(c.mu);
    c.idle.emplace(b.bytes, b);
    c.idle_bytes += b.bytes;
}
}  // namespace

void cache_free(void *p) { cache_release(p, false, nullptr); }
void cache_free(void *p, cudaStream_t last_use) { cache_release(p, true, last_use); }

cufsp_status ReduceScratch::init(int ctas, int k) {
    release();
    max_ctas = ctas;
    max_k = k;
    CUFSP_CUDA_TRY(cache_alloc((void **)&partials, sizeof(double) * (size_t)ctas * k));
    CUFSP_CUDA_TRY(cache_alloc((void **)&counter, sizeof(unsigned int) * 4));
    CUFSP_CUDA_TRY(cudaMemset(counter, 0, sizeof(unsigned int) * 4));
    CUFSP_CUDA_TRY(upload_fence());
    return CUFSP_SUCCESS;
}

cufsp_status ReduceScratch::init(int ctas, int k, cudaStream_t st) {
    release();
    max_ctas = ctas;
    max_k = k;
    CUFSP_CUDA_TRY(cache_alloc((void **)&partials, sizeof(double) * (size_t)ctas * k));
    CUFSP_CUDA_TRY(cache_alloc((void **)&counter, sizeof(unsigned int) * 4));
    CUFSP_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned int) * 4, st));
    return CUFSP_SUCCESS;
}

void ReduceScratch::release() {
    cache_free(partials);
    cache_free(counter);
    partials = nullptr;
    counter = nullptr;
}

void ReduceScratch::release(cudaStream_t last_use) {
    cache_free(partials, last_use);
    cache_free(counter, last_use);
    partials = nullptr;
    counter = nullptr;
}

// ---- kernels ---------------------------------------------------------------------------------

struct DecodeArgs {
    int ns;
    FastDiv div[CUFSP_MAX_SPECIES];
};

// fsp_get_states (src/cme_util.cu:24-41).  Each CTA decodes 256 consecutive states into shared
// memory and writes them out as one contiguous, coalesced block of 256*ns ints.
__global__ void __launch_bounds__(256) k_get_states(DecodeArgs a, int n, int *__restrict__ out) {
    extern __shared__ int sm_states[];
    const int64_t base = (int64_t)blockIdx.x * 256;
    const int i = (int)(base + threadIdx.x);
    if (i < n) {
        uint32_t rem = (uint32_t)i;
        for (int s = 0; s < a.ns; ++s) {
            uint32_t q = fd_div(rem, a.div[s]);
            sm_states[threadIdx.x * a.ns + s] = (int)(rem - q * a.div[s].d);
            rem = q;
        }
    }
    __syncthreads();
    const int64_t count = min((int64_t)256, (int64_t)n - base) * a.ns;
    int *dst = out + base * a.ns;
    for (int t = threadIdx.x; t < count; t += 256) dst[t] = sm_states[t];
}

template <int KP>
__global__ void __launch_bounds__(kRedThreads) k_sum(int64_t n, const double *__restrict__ x, bool squares,
                                                     double *__restrict__ partials, unsigned int *__restrict__ counter,
                                                     double *__restrict__ out) {
    __shared__ RedSmem<KP> sm;
    double acc[KP] = {0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double v = x[i];
        acc[0] += squares ? v * v : v;
    }
    if (grid_reduce<KP>(acc, 1, partials, counter, sm) && threadIdx.x == 0)
        out[0] = squares ? sqrt(sm.final_[0]) : sm.final_[0];
}

__global__ void k_fill(int64_t n, double *__restrict__ x, double v) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] = v;
}

__global__ void k_scale(int64_t n, double *__restrict__ x, const double *__restrict__ d_alpha, double alpha) {
    const double a = alpha * (d_alpha ? d_alpha[0] : 1.0);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] *= a;
}

static int max_stream_ctas() { return device_info().sm_count * 4; }

cufsp_status launch_sum(int64_t n, const double *x, double *d_out, ReduceScratch &rs, cudaStream_t st) {
    int g = stream_grid(n, 4, std::min(max_stream_ctas(), rs.max_ctas));
    k_sum<1><<<g, kRedThreads, 0, st>>>(n, x, false, rs.partials, rs.counter, d_out);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

cufsp_status launch_nrm2(int64_t n, const double *x, double *d_out, ReduceScratch &rs, cudaStream_t st) {
    int g = stream_grid(n, 4, std::min(max_stream_ctas(), rs.max_ctas));
    k_sum<1><<<g, kRedThreads, 0, st>>>(n, x, true, rs.partials, rs.counter, d_out);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

cufsp_status launch_fill(int64_t n, double *x, double v, cudaStream_t st) {
    int g = stream_grid(n, 4, max_stream_ctas());
    k_fill<<<g, 256, 0, st>>>(n, x, v);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

cufsp_status launch_scale(int64_t n, double *x, const double *d_alpha, double alpha, cudaStream_t st) {
    int g = stream_grid(n, 4, max_stream_ctas());
    k_scale<<<g, 256, 0, st>>>(n, x, d_alpha, alpha);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

// ---- model validation -------------------------------------------------------------------------

cufsp_status model_from_desc(const cufsp_model_desc *d, bool need_tables, ModelHost &m, bool external_table) {
    if (!d) return set_error(CUFSP_ERR_INVALID_ARG, "model descriptor is NULL");
    if (d->n_species < 1 || d->n_species > CUFSP_MAX_SPECIES)
        return set_error(CUFSP_ERR_INVALID_ARG, "n_species must be in [1, 16]");
    if (d->n_reactions < 1 || d->n_reactions > CUFSP_MAX_REACTIONS_SPARSE)
        return set_error(CUFSP_ERR_INVALID_ARG, "n_reactions must be in [1, 256]");
    if (!d->fsp_bounds || !d->stoich_vals || !d->stoich_colidxs || !d->stoich_rowptrs)
        return set_error(CUFSP_ERR_INVALID_ARG, "fsp_bounds and the stoichiometry CSR arrays are required");
    m.ns = d->n_species;
    m.nr = d->n_reactions;
    m.bounds.assign(d->fsp_bounds, d->fsp_bounds + m.ns);
    int64_t n = 1;
    for (int s = 0; s < m.ns; ++s) {
        if (m.bounds[s] < 0) return set_error(CUFSP_ERR_INVALID_ARG, "fsp_bounds must be >= 0");
        n *= (int64_t)m.bounds[s] + 1;
        if (n > 2147483647LL)
            return set_error(CUFSP_ERR_OVERFLOW, "number of states exceeds 2^31-1 (int32 state index)");
    }
    m.n = n;
    m.nu.assign((size_t)m.nr * m.ns, 0);
    if (d->stoich_rowptrs[0] != 0) return set_error(CUFSP_ERR_INVALID_ARG, "stoich_rowptrs[0] must be 0");
    for (int r = 0; r < m.nr; ++r) {
        int a = d->stoich_rowptrs[r], b = d->stoich_rowptrs[r + 1];
        if (b < a) return set_error(CUFSP_ERR_INVALID_ARG, "stoich_rowptrs must be non-decreasing");
        for (int i = a; i < b; ++i) {
            int c = d->stoich_colidxs[i];
            if (c < 0 || c >= m.ns) return set_error(CUFSP_ERR_INVALID_ARG, "stoich column index out of range");
            m.nu[(size_t)r * m.ns + c] += d->stoich_vals[i];
        }
    }
    m.tab_off.resize(m.ns);
    int off = 0;
    for (int s = 0; s < m.ns; ++s) {
        m.tab_off[s] = off;
        off += m.bounds[s] + 1;
    }
    m.tab_stride = off;
    m.prop_device = d->prop_device;
    m.tcoef = d->tcoef;
    m.tcoef_user = d->tcoef_user;
    const size_t tsz = (size_t)m.nr * m.tab_stride;
    if (d->factor_tables) {
        m.tables.assign(d->factor_tables, d->factor_tables + tsz);
    } else if (d->prop_factor) {
        // fspmat_sdkron_fill_host_data (src/fspmat_kron_kernels.cu:170-190): f_{r,s}(0..b_s)
        m.tables.resize(tsz);
        size_t iv = 0;
        for (int r = 0; r < m.nr; ++r)
            for (int s = 0; s < m.ns; ++s)
                for (int x = 0; x <= m.bounds[s]; ++x) m.tables[iv++] = d->prop_factor(x, s, r);
    }
    for (double v : m.tables)
        if (!std::isfinite(v)) return set_error(CUFSP_ERR_NONFINITE, "propensity factor table holds NaN/Inf");
    if (need_tables && m.tables.empty())
        return set_error(CUFSP_ERR_INVALID_ARG, "KRONECKER format needs factor_tables or prop_factor");
    if (m.tables.empty() && !m.prop_device && !external_table)
        return set_error(CUFSP_ERR_INVALID_ARG, "no propensity source (factor_tables, prop_factor or prop_device)");
    return CUFSP_SUCCESS;
}

}  // namespace cufsp

using namespace cufsp;

// ---- C ABI: status and indexing --------------------------------------------------------------

extern "C" cufsp_status cufsp_cache_trim(size_t *freed_bytes) {
    const size_t f = cufsp::cache_trim_all();
    if (freed_bytes) *freed_bytes = f;
    return CUFSP_SUCCESS;
}

extern "C" const char *cufsp_status_string(cufsp_status s) {
    switch (s) {
        case CUFSP_SUCCESS: return "CUFSP_SUCCESS";
        case CUFSP_ERR_INVALID_ARG: return "CUFSP_ERR_INVALID_ARG";
        case CUFSP_ERR_OVERFLOW: return "CUFSP_ERR_OVERFLOW";
        case CUFSP_ERR_ALLOC: return "CUFSP_ERR_ALLOC";
        case CUFSP_ERR_CUDA: return "CUFSP_ERR_CUDA";
        case CUFSP_ERR_NONFINITE: return "CUFSP_ERR_NONFINITE";
        case CUFSP_ERR_STEP_LIMIT: return "CUFSP_ERR_STEP_LIMIT";
        case CUFSP_ERR_UNSUPPORTED: return "CUFSP_ERR_UNSUPPORTED";
        case CUFSP_ERR_NO_DEVICE: return "CUFSP_ERR_NO_DEVICE";
    }
    return "CUFSP_ERR_UNKNOWN";
}

extern "C" const char *cufsp_last_error(void) { return g_last_error.c_str(); }

extern "C" cufsp_status cufsp_num_states(int ns, const int *bounds, int64_t *n_states) {
    if (!bounds || !n_states || ns < 1) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_num_states: bad argument");
    int64_t n = 1;
    for (int s = 0; s < ns; ++s) {
        if (bounds[s] < 0) return set_error(CUFSP_ERR_INVALID_ARG, "fsp_bounds must be >= 0");
        n *= (int64_t)bounds[s] + 1;
        if (n > ((int64_t)1 << 62)) return set_error(CUFSP_ERR_OVERFLOW, "state count overflow");
    }
    *n_states = n;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_indx2state(int64_t indx, int *state, int ns, const int *bounds) {
    if (!state || !bounds || ns < 1 || indx < 0) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_indx2state: bad argument");
    for (int s = 0; s < ns; ++s) {
        int64_t d = (int64_t)bounds[s] + 1;
        state[s] = (int)(indx % d);
        indx /= d;
    }
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_state2indx(const int *state, int ns, const int *bounds, int64_t *indx) {
    if (!state || !bounds || !indx || ns < 1) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_state2indx: bad argument");
    int64_t id = 0, np = 1;
    for (int s = 0; s < ns; ++s) {
        if (state[s] < 0 || state[s] > bounds[s]) return set_error(CUFSP_ERR_INVALID_ARG, "state outside the FSP box");
        id += (int64_t)state[s] * np;
        np *= (int64_t)bounds[s] + 1;
    }
    *indx = id;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_get_states(int ns, const int *bounds, int *d_states, cufsp_stream_t stream) {
    if (!bounds || !d_states || ns < 1 || ns > CUFSP_MAX_SPECIES)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_get_states: bad argument");
    int64_t n = 0;
    cufsp_status s = cufsp_num_states(ns, bounds, &n);
    if (s != CUFSP_SUCCESS) return s;
    if (n > 2147483647LL) return set_error(CUFSP_ERR_OVERFLOW, "number of states exceeds 2^31-1");
    DecodeArgs a;
    a.ns = ns;
    for (int k = 0; k < ns; ++k) a.div[k] = make_fastdiv((uint32_t)bounds[k] + 1u);
    int64_t grid = (n + 255) / 256;
    k_get_states<<<(unsigned)grid, 256, 256 * ns * sizeof(int), (cudaStream_t)stream>>>(a, (int)n, d_states);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_vec_sum(int64_t n, const double *x, double *out, cufsp_stream_t stream) {
    if (!x || !out || n < 0) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_vec_sum: bad argument");
    ReduceScratch rs;
    cufsp_status s = rs.init(device_info().sm_count * 4, 1);
    if (s != CUFSP_SUCCESS) { rs.release(); return s; }
    double *d_out = nullptr;
    if (dev_malloc(&d_out, sizeof(double)) != cudaSuccess) { rs.release(); return set_error(CUFSP_ERR_ALLOC, "cudaMalloc"); }
    s = launch_sum(n, x, d_out, rs, (cudaStream_t)stream);
    if (s == CUFSP_SUCCESS) {
        cudaError_t e = cudaMemcpyAsync(out, d_out, sizeof(double), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
        if (e != cudaSuccess) s = cuda_error(e, "cufsp_vec_sum");
    }
    cudaFree(d_out);
    rs.release();
    return s;
}
