// cufsp_batch.cu -- host side of the batched persistent Krylov solver (kernel: cufsp_batch.cuh).
//
// Many FSP instances of one reaction network -- different boxes, factor tables and rate
// coefficients -- are solved to a common final time in one persistent launch of thread-block
// clusters.  At create time the network's pattern (stoichiometry, and per reaction and species
// whether the factor table is 1, the identity x or a general table in every instance) is written
// as an NVRTC prefix and the kernel is compiled for sm_100a.  Launch shapes (CTAs per cluster,
// threads per CTA) come from a project-written autotuner that times candidate shapes on a sample of
// the batch and keeps the winner in an in-process table and in a small cache file.  Each solve is
// replayed as a CUDA graph (work-counter reset + the persistent kernel).
#include <nvrtc.h>
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "cufsp_internal.h"
#include "cufsp_batch.cuh"

namespace cufsp {
namespace {

const char *kBatchSource =
#include "cufsp_batch_src.inc"
    ;

struct BatchKernel {
    cudaLibrary_t lib = nullptr;
    cudaKernel_t k = nullptr;
    int smem = 0;
};

std::mutex g_batch_mu;
std::map<std::string, std::shared_ptr<BatchKernel>> g_batch_cache;
struct Shape {
    int cluster, threads, minb;
};
std::map<std::string, Shape> g_tune_cache;  // key -> launch shape

int env_int(const char *name, int dflt) {
    const char *v = getenv(name);
    return v ? atoi(v) : dflt;
}

// NVRTC compile of one batched-kernel source to a cubin (no lock: NVRTC programs are independent, so
// the autotuner compiles its candidate sources on parallel host threads).
bool compile_cubin(const std::string &src, std::vector<char> &cubin, std::string &why) {
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), "cufsp_batch.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
        why = "nvrtcCreateProgram failed";
        return false;
    }
    const char *opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--fmad=true", "-lineinfo",
                          "-I/usr/local/cuda/include"};
    const nvrtcResult rc = nvrtcCompileProgram(prog, 5, opts);
    if (rc != NVRTC_SUCCESS) {
        size_t ls = 0;
        nvrtcGetProgramLogSize(prog, &ls);
        std::string log(ls, '\0');
        if (ls > 1) nvrtcGetProgramLog(prog, &log[0]);
        why = std::string("NVRTC: ") + nvrtcGetErrorString(rc) + ": " + log.substr(0, 3000);
        nvrtcDestroyProgram(&prog);
        return false;
    }
    size_t cs = 0;
    cubin.clear();
    if (nvrtcGetCUBINSize(prog, &cs) == NVRTC_SUCCESS && cs > 0) {
        cubin.resize(cs);
        if (nvrtcGetCUBIN(prog, cubin.data()) != NVRTC_SUCCESS) cubin.clear();
    }
    nvrtcDestroyProgram(&prog);
    if (cubin.empty()) {
        why = "NVRTC produced no cubin";
        return false;
    }
    return true;
}

// Loads a compiled cubin into the process-wide kernel cache (caller holds g_batch_mu).
std::shared_ptr<BatchKernel> load_kernel_locked(const std::string &src, const std::vector<char> &cubin,
                                                std::string &why) {
    auto it = g_batch_cache.find(src);
    if (it != g_batch_cache.end()) return it->second;
    auto bk = std::make_shared<BatchKernel>();
    cudaError_t e = cudaLibraryLoadData(&bk->lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&bk->k, bk->lib, "cufsp_batch_expv");
    void *dptr = nullptr;
    size_t bytes = 0;
    if (e == cudaSuccess) e = cudaLibraryGetGlobal(&dptr, &bytes, bk->lib, "cufsp_batch_smem_bytes");
    if (e == cudaSuccess) e = cudaMemcpy(&bk->smem, dptr, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute((const void *)bk->k, cudaFuncAttributeMaxDynamicSharedMemorySize, bk->smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute((const void *)bk->k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) {
        cudaGetLastError();
        why = std::string("loading the batched kernel: ") + cudaGetErrorString(e);
        return nullptr;
    }
    g_batch_cache[src] = bk;
    return bk;
}

std::shared_ptr<BatchKernel> batch_kernel(const std::string &src, std::string &why) {
    std::lock_guard<std::mutex> lock(g_batch_mu);
    auto it = g_batch_cache.find(src);
    if (it != g_batch_cache.end()) return it->second;
    std::vector<char> cubin;
    if (!compile_cubin(src, cubin, why)) return nullptr;
    return load_kernel_locked(src, cubin, why);
}

// Compiles the sources not yet in the kernel cache on one host thread each and loads them.
void prefetch_kernels(const std::vector<std::string> &srcs) {
    std::vector<std::string> todo;
    {
        std::lock_guard<std::mutex> lock(g_batch_mu);
        for (const std::string &s : srcs)
            if (!g_batch_cache.count(s) && std::find(todo.begin(), todo.end(), s) == todo.end()) todo.push_back(s);
    }
    if (todo.size() < 2) return;  // nothing to overlap; batch_kernel compiles on demand
    std::vector<std::vector<char>> cubins(todo.size());
    std::vector<std::string> why(todo.size());
    std::vector<char> ok(todo.size(), 0);
    std::vector<std::thread> th;
    for (size_t i = 0; i < todo.size(); ++i)
        th.emplace_back([&, i] { ok[i] = compile_cubin(todo[i], cubins[i], why[i]); });
    for (auto &t : th) t.join();
    std::lock_guard<std::mutex> lock(g_batch_mu);
    for (size_t i = 0; i < todo.size(); ++i)
        if (ok[i]) load_kernel_locked(todo[i], cubins[i], why[i]);  // failures recompile (and report) on demand
}

void emit_fn2(std::ostringstream &s, const char *name, const std::vector<int> &v, int ns) {
    s << "__host__ __device__ __forceinline__ constexpr int " << name << "(int r, int sp) {";
    for (size_t i = 0; i < v.size(); ++i)
        if (v[i] != 0) s << " if (r == " << i / ns << " && sp == " << i % ns << ") return " << v[i] << ";";
    s << " return 0; }\n";
}

std::string cache_path() {
    if (const char *p = getenv("CUFSP_AUTOTUNE_CACHE")) return p;
    const char *home = getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/cufsp_batch_autotune.txt";
}

bool cache_lookup(const std::string &key, Shape &sh) {
    std::lock_guard<std::mutex> lock(g_batch_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
        sh = it->second;
        return true;
    }
    std::ifstream f(cache_path());
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream ls(line);
        std::string k;
        Shape s2{0, 0, 0};
        if (ls >> k >> s2.cluster >> s2.threads >> s2.minb && k == key && s2.cluster > 0 && s2.threads > 0 &&
            s2.minb > 0) {
            g_tune_cache[key] = s2;
            sh = s2;
            return true;
        }
    }
    return false;
}

void cache_store(const std::string &key, const Shape &sh, double ms) {
    std::lock_guard<std::mutex> lock(g_batch_mu);
    g_tune_cache[key] = sh;
    const std::string path = cache_path();
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos && slash > 0) mkdir(path.substr(0, slash).c_str(), 0755);  // one level
    std::ofstream f(path, std::ios::app);
    if (f) f << key << " " << sh.cluster << " " << sh.threads << " " << sh.minb << " " << ms << "\n";
}

}  // namespace
}  // namespace cufsp

using namespace cufsp;

struct cufsp_batch_s {
    int ns = 0, nr = 0, n_inst = 0, m = 30, iop = 0, q_iop = 2;
    double tol = 1e-8, anorm = 1.0;
    int max_steps = 100000, max_reject = 1000;
    std::vector<int> nu;                   // [nr][ns]
    std::vector<int> kinds;                // [nr][ns]
    std::vector<CufspBatchInst> inst;      // host copy of the descriptors
    std::vector<int64_t> offsets;          // packed layout, n_inst + 1
    std::vector<int> order;                // largest first
    int64_t n_max = 0;
    std::string pattern;                   // NVRTC prefix without the launch shape
    CufspBatchInst *d_inst = nullptr;
    int *d_order = nullptr, *d_order_sample = nullptr;
    int n_sample = 0;
    double *d_tables = nullptr;
    CufspBatchStat *d_stats = nullptr;
    unsigned *d_counter = nullptr;
    double *d_work = nullptr;
    size_t work_doubles = 0;
    double *d_scratch = nullptr;           // autotuner trial vectors
    // chosen launch shape
    int cluster = 0, threads = 0, minb = 1;
    std::shared_ptr<BatchKernel> kern;
    int n_clusters = 0;
    double tuned_ms = 0.0;
    double tune_s = 0.0;                   // wall time of the autotuner (compiles and trial launches)
    double tune_compile_s = 0.0;           // of which compiling the candidate shapes
    bool tuned = false;
    // graph of the last solve
    cudaGraphExec_t gexec = nullptr;
    double g_tfinal = -1.0;
    double *g_p = nullptr;
    cudaStream_t g_stream = nullptr;
    std::string describe;
};

namespace {

// Launch shape: CTAs per cluster, threads per CTA, CTAs per SM promised to the compiler (register cap).
std::string shape_source(const cufsp_batch *B, int threads, int minb) {
    std::ostringstream s;
    s << "#define CUFSP_BATCH_THREADS " << threads << "\n#define CUFSP_BATCH_MINB " << minb << "\n" << B->pattern;
    return s.str() + kBatchSource;
}

// Grid (clusters) for a shape; 0 when the shape does not fit.
int clusters_for(cufsp_batch *B, const BatchKernel &k, int cluster, int threads) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cluster * 64);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = k.smem;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, (const void *)k.k, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return std::min(n, B->n_inst);
}

cufsp_status ensure_work(cufsp_batch *B, int n_clusters) {
    const size_t need = (size_t)n_clusters * (size_t)(B->m + 1) * (size_t)B->n_max;
    if (need <= B->work_doubles) return CUFSP_SUCCESS;
    if (B->d_work) cudaFree(B->d_work);
    B->d_work = nullptr;
    B->work_doubles = 0;
    CUFSP_CUDA_TRY(dev_malloc(&B->d_work, sizeof(double) * need));
    B->work_doubles = need;
    return CUFSP_SUCCESS;
}

cufsp_status launch(cufsp_batch *B, const BatchKernel &k, int cluster, int threads, int n_clusters, double t_final,
                    double *p, const int *order, int n_inst, cudaStream_t st) {
    CufspBatchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.inst = B->d_inst;
    a.order = order;
    a.tables = B->d_tables;
    a.p = p;
    a.work = B->d_work;
    a.work_stride = (long long)(B->m + 1) * B->n_max;
    a.counter = B->d_counter;
    a.stats = B->d_stats;
    a.n_inst = n_inst;
    a.max_steps = B->max_steps;
    a.max_reject = B->max_reject;
    a.t_final = t_final;
    a.tol = B->tol;
    a.anorm = B->anorm;
    CUFSP_CUDA_TRY(cudaMemsetAsync(B->d_counter, 0, sizeof(unsigned), st));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)(cluster * n_clusters));
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = k.smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {&a};
    CUFSP_CUDA_TRY(cudaLaunchKernelExC(&cfg, (const void *)k.k, args));
    return CUFSP_SUCCESS;
}

std::string describe_shape(const cufsp_batch *B) {
    std::ostringstream d;
    d << "batched Krylov (NVRTC, sm_100a, one persistent launch): " << B->n_inst << " instances, m=" << B->m
      << (B->iop ? " IOP" : "") << ", " << B->n_clusters << " clusters x " << B->cluster << " CTAs x " << B->threads
      << " threads (" << B->minb << " CTA/SM bound), smem " << B->kern->smem << " B/CTA";
    if (B->tune_s > 0.0)
        d << "; autotuner " << std::fixed << std::setprecision(1) << B->tune_s << " s on " << B->n_sample
          << " instances (compiles " << B->tune_compile_s << " s)";
    return d.str();
}

std::string tune_key(const cufsp_batch *B) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp p;
    cudaGetDeviceProperties(&p, dev);
    std::string name = p.name;
    std::replace(name.begin(), name.end(), ' ', '_');
    const size_t h = std::hash<std::string>{}(B->pattern);
    // size class: log2 of the largest instance and of the instance count
    std::ostringstream k;
    k << name << "|" << std::hex << h << std::dec << "|n" << (int)std::log2((double)B->n_max) << "|b"
      << (int)std::log2((double)B->n_inst);
    return k.str();
}

// Autotuner: time each candidate launch shape on a sample of the batch (copies of the caller's
// vectors) over a thirty-second of the requested horizon (a few Krylov steps per instance: the cost
// per step, not the horizon, separates the shapes) and keep the fastest.
cufsp_status autotune(cufsp_batch *B, double t_final, const double *p, cudaStream_t st) {
    const std::string key = tune_key(B);
    Shape sh{env_int("CUFSP_BATCH_CLUSTER", 0), env_int("CUFSP_BATCH_THREADS", 0), env_int("CUFSP_BATCH_MINB", 1)};
    std::string why;
    if (sh.cluster > 0 && sh.threads > 0) {
        B->cluster = sh.cluster;
        B->threads = sh.threads;
        B->minb = std::max(1, sh.minb);
    } else if (cache_lookup(key, sh)) {
        B->cluster = sh.cluster;
        B->threads = sh.threads;
        B->minb = sh.minb;
    } else {
        // (16 x 256 ran within 1 % of 8 x 256 on full batches and is not timed)
        const Shape cands[] = {{8, 256, 1}, {4, 512, 1}, {8, 512, 1}, {16, 512, 1}, {8, 256, 2}};
        const auto t_tune = std::chrono::steady_clock::now();
        {
            std::vector<std::string> srcs;
            for (const Shape &cd : cands) srcs.push_back(shape_source(B, cd.threads, cd.minb));
            prefetch_kernels(srcs);
        }
        B->tune_compile_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_tune).count();
        const int64_t total = B->offsets.back();
        if (!B->d_scratch) CUFSP_CUDA_TRY(dev_malloc(&B->d_scratch, sizeof(double) * (size_t)total));
        double best = 1e300;
        cudaEvent_t e0, e1;
        CUFSP_CUDA_TRY(cudaEventCreate(&e0));
        CUFSP_CUDA_TRY(cudaEventCreate(&e1));
        for (const Shape &cd : cands) {
            auto k = batch_kernel(shape_source(B, cd.threads, cd.minb), why);
            if (!k) continue;
            const int ncl = clusters_for(B, *k, cd.cluster, cd.threads);
            if (ncl < 1) continue;
            if (ensure_work(B, ncl) != CUFSP_SUCCESS) continue;
            CUFSP_CUDA_TRY(cudaMemcpyAsync(B->d_scratch, p, sizeof(double) * (size_t)total, cudaMemcpyDeviceToDevice, st));
            CUFSP_CUDA_TRY(cudaEventRecord(e0, st));
            cufsp_status s = launch(B, *k, cd.cluster, cd.threads, ncl, t_final / 32.0, B->d_scratch, B->d_order_sample,
                                    B->n_sample, st);
            CUFSP_CUDA_TRY(cudaEventRecord(e1, st));
            if (s != CUFSP_SUCCESS || cudaStreamSynchronize(st) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) {
                best = ms;
                B->cluster = cd.cluster;
                B->threads = cd.threads;
                B->minb = cd.minb;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (B->cluster == 0) return set_error(CUFSP_ERR_CUDA, "batched solver: no launch shape fits this device: " + why);
        B->tuned_ms = best;
        B->tune_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_tune).count();
        cache_store(key, Shape{B->cluster, B->threads, B->minb}, best);
    }
    B->kern = batch_kernel(shape_source(B, B->threads, B->minb), why);
    if (!B->kern) return set_error(CUFSP_ERR_CUDA, "batched solver: " + why);
    B->n_clusters = clusters_for(B, *B->kern, B->cluster, B->threads);
    if (B->n_clusters < 1) return set_error(CUFSP_ERR_UNSUPPORTED, "batched solver: launch shape does not fit");
    cufsp_status s = ensure_work(B, B->n_clusters);
    if (s != CUFSP_SUCCESS) return s;
    B->tuned = true;
    B->describe = describe_shape(B);
    return CUFSP_SUCCESS;
}

}  // namespace

extern "C" cufsp_status cufsp_batch_create(const cufsp_batch_desc *d, int m, double tol, int iop, int q_iop,
                                           cufsp_batch **out) {
    clear_error();
    if (!out || !d) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_create: NULL argument");
    *out = nullptr;
    if (d->n_species < 1 || d->n_species > CUFSP_BATCH_MAXS)
        return set_error(CUFSP_ERR_UNSUPPORTED, "cufsp_batch_create: 1..8 species supported");
    if (d->n_reactions < 1 || d->n_reactions > CUFSP_BATCH_MAXR)
        return set_error(CUFSP_ERR_UNSUPPORTED, "cufsp_batch_create: 1..32 reactions supported");
    if (d->n_instances < 1 || !d->fsp_bounds || !d->factor_tables || !d->coefs || !d->stoich_rowptrs ||
        !d->stoich_colidxs || !d->stoich_vals)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_create: incomplete description");
    if (m < 1 || m > 32) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_create: m must be in [1, 32]");
    if (!(tol > 0.0)) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_create: tol must be > 0");
    if (iop && q_iop < 1) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_create: q_iop must be >= 1");
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
        cudaGetLastError();
        return set_error(CUFSP_ERR_NO_DEVICE, "no CUDA device available");
    }
    std::unique_ptr<cufsp_batch> B(new cufsp_batch());
    const int ns = d->n_species, nr = d->n_reactions, ni = d->n_instances;
    B->ns = ns;
    B->nr = nr;
    B->n_inst = ni;
    B->m = m;
    B->tol = tol;
    B->iop = iop ? 1 : 0;
    B->q_iop = q_iop;
    B->nu.assign((size_t)nr * ns, 0);
    for (int r = 0; r < nr; ++r)
        for (int k = d->stoich_rowptrs[r]; k < d->stoich_rowptrs[r + 1]; ++k) {
            const int sp = d->stoich_colidxs[k];
            if (sp < 0 || sp >= ns) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_create: bad stoichiometry column");
            B->nu[(size_t)r * ns + sp] += d->stoich_vals[k];
        }
    // per instance: box, offsets, tables; factor kinds over all instances
    B->kinds.assign((size_t)nr * ns, 0);
    std::vector<int> is_one((size_t)nr * ns, 1), is_id((size_t)nr * ns, 1);
    B->inst.resize(ni);
    B->offsets.assign(ni + 1, 0);
    std::vector<int64_t> tab_off_inst(ni + 1, 0);
    for (int i = 0; i < ni; ++i) {
        CufspBatchInst &I = B->inst[i];
        std::memset(&I, 0, sizeof(I));
        int64_t n = 1, stride = 1, tsz = 0;
        std::vector<int64_t> strides(ns);
        for (int sp = 0; sp < ns; ++sp) {
            const int b = d->fsp_bounds[(size_t)i * ns + sp];
            if (b < 0) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_create: negative bound");
            I.dims[sp] = b + 1;
            I.tab_off[sp] = (int)tsz;
            tsz += b + 1;
            strides[sp] = stride;
            stride *= (b + 1);
            n *= (b + 1);
            if (n > 2147483647LL) return set_error(CUFSP_ERR_OVERFLOW, "cufsp_batch_create: an instance exceeds 2^31 states");
            const FastDiv f = make_fastdiv((uint32_t)(b + 1));
            I.div[sp].d = f.d;
            I.div[sp].mul = f.mul;
            I.div[sp].shift = f.shift;
        }
        I.n = (int)n;
        I.tab_stride = (int)tsz;
        for (int r = 0; r < nr; ++r) {
            int64_t dl = 0;
            for (int sp = 0; sp < ns; ++sp) dl += (int64_t)B->nu[(size_t)r * ns + sp] * strides[sp];
            I.delta[r] = (int)dl;
            const double c = d->coefs[(size_t)i * nr + r];
            if (!std::isfinite(c)) return set_error(CUFSP_ERR_NONFINITE, "cufsp_batch_create: coefficient is NaN/Inf");
            I.coef[r] = c;
        }
        const double *tb = d->factor_tables[i];
        if (!tb) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_create: NULL factor table");
        for (int r = 0; r < nr; ++r)
            for (int sp = 0; sp < ns; ++sp)
                for (int x = 0; x < I.dims[sp]; ++x) {
                    const double v = tb[(size_t)r * tsz + I.tab_off[sp] + x];
                    if (!std::isfinite(v)) return set_error(CUFSP_ERR_NONFINITE, "cufsp_batch_create: factor table holds NaN/Inf");
                    if (v != 1.0) is_one[(size_t)r * ns + sp] = 0;
                    if (v != (double)x) is_id[(size_t)r * ns + sp] = 0;
                }
        I.off = B->offsets[i];
        B->offsets[i + 1] = B->offsets[i] + ((n + 1) & ~int64_t(1));  // 16-byte aligned vectors
        I.tab = tab_off_inst[i];
        tab_off_inst[i + 1] = tab_off_inst[i] + (int64_t)nr * tsz;
        B->n_max = std::max<int64_t>(B->n_max, n);
    }
    for (size_t k = 0; k < B->kinds.size(); ++k) B->kinds[k] = is_one[k] ? 0 : (is_id[k] ? 1 : 2);
    B->order.resize(ni);
    std::iota(B->order.begin(), B->order.end(), 0);
    std::stable_sort(B->order.begin(), B->order.end(), [&](int a, int b) { return B->inst[a].n > B->inst[b].n; });
    // autotuner sample: every k-th instance of the size-sorted order, up to 96 -- more instances than
    // any candidate shape has clusters (148 SMs in clusters of 4 CTAs at 2 CTAs per SM: 74), so that
    // every candidate is timed with all of its clusters busy, as in the full batch
    constexpr int kSampleMax = 96;
    std::vector<int> sample;
    const int stride_s = std::max(1, ni / kSampleMax);
    for (int i = 0; i < ni && (int)sample.size() < kSampleMax; i += stride_s) sample.push_back(B->order[i]);
    B->n_sample = (int)sample.size();

    std::ostringstream s;
    s << "#define CUFSP_BATCH_NS " << ns << "\n#define CUFSP_BATCH_NR " << nr << "\n#define CUFSP_BATCH_M " << m
      << "\n#define CUFSP_BATCH_IOP " << B->iop << "\n#define CUFSP_BATCH_QIOP " << q_iop << "\nnamespace cufsp_batch {\n";
    emit_fn2(s, "nu", B->nu, ns);
    emit_fn2(s, "kind", B->kinds, ns);
    s << "}\n";
    B->pattern = s.str();

    std::vector<double> tabs((size_t)tab_off_inst[ni]);
    for (int i = 0; i < ni; ++i)
        std::memcpy(tabs.data() + tab_off_inst[i], d->factor_tables[i],
                    sizeof(double) * (size_t)(tab_off_inst[i + 1] - tab_off_inst[i]));
    cudaError_t e = dev_malloc(&B->d_inst, sizeof(CufspBatchInst) * ni);
    if (e == cudaSuccess) e = dev_malloc(&B->d_order, sizeof(int) * ni);
    if (e == cudaSuccess) e = dev_malloc(&B->d_order_sample, sizeof(int) * B->n_sample);
    if (e == cudaSuccess) e = dev_malloc(&B->d_tables, sizeof(double) * std::max<size_t>(1, tabs.size()));
    if (e == cudaSuccess) e = dev_malloc(&B->d_stats, sizeof(CufspBatchStat) * ni);
    if (e == cudaSuccess) e = dev_malloc(&B->d_counter, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemcpy(B->d_inst, B->inst.data(), sizeof(CufspBatchInst) * ni, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(B->d_order, B->order.data(), sizeof(int) * ni, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(B->d_order_sample, sample.data(), sizeof(int) * B->n_sample, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !tabs.empty())
        e = cudaMemcpy(B->d_tables, tabs.data(), sizeof(double) * tabs.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(B->d_stats, 0, sizeof(CufspBatchStat) * ni);
    if (e == cudaSuccess) e = upload_fence();
    if (e != cudaSuccess) {
        cufsp_batch_destroy(B.release());
        return cuda_error(e, "cufsp_batch_create");
    }
    // compile the default shape now so that a bad network fails at create
    std::string why;
    if (!batch_kernel(shape_source(B.get(), 256, 1), why)) {
        cufsp_batch_destroy(B.release());
        return set_error(CUFSP_ERR_CUDA, "cufsp_batch_create: " + why);
    }
    *out = B.release();
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_batch_destroy(cufsp_batch *B) {
    if (!B) return CUFSP_SUCCESS;
    if (B->gexec) cudaGraphExecDestroy(B->gexec);
    if (B->d_inst) cudaFree(B->d_inst);
    if (B->d_order) cudaFree(B->d_order);
    if (B->d_order_sample) cudaFree(B->d_order_sample);
    if (B->d_tables) cudaFree(B->d_tables);
    if (B->d_stats) cudaFree(B->d_stats);
    if (B->d_counter) cudaFree(B->d_counter);
    if (B->d_work) cudaFree(B->d_work);
    if (B->d_scratch) cudaFree(B->d_scratch);
    delete B;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_batch_layout(const cufsp_batch *B, int64_t *offsets) {
    if (!B || !offsets) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_layout: NULL argument");
    std::copy(B->offsets.begin(), B->offsets.end(), offsets);
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_batch_set_limits(cufsp_batch *B, int max_steps, int max_reject) {
    if (!B || max_steps < 1 || max_reject < 1) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_set_limits: bad argument");
    B->max_steps = max_steps;
    B->max_reject = max_reject;
    if (B->gexec) {
        cudaGraphExecDestroy(B->gexec);
        B->gexec = nullptr;
    }
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_batch_set_coefs(cufsp_batch *B, const double *coefs) {
    if (!B || !coefs) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_set_coefs: NULL argument");
    for (int i = 0; i < B->n_inst; ++i)
        for (int r = 0; r < B->nr; ++r) {
            const double c = coefs[(size_t)i * B->nr + r];
            if (!std::isfinite(c)) return set_error(CUFSP_ERR_NONFINITE, "cufsp_batch_set_coefs: NaN/Inf");
            B->inst[i].coef[r] = c;
        }
    CUFSP_CUDA_TRY(cudaMemcpy(B->d_inst, B->inst.data(), sizeof(CufspBatchInst) * B->n_inst, cudaMemcpyHostToDevice));
    CUFSP_CUDA_TRY(upload_fence());
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_batch_set_shape(cufsp_batch *B, int cluster_ctas, int threads) {
    if (!B) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_set_shape: NULL argument");
    if (cluster_ctas == 0 && threads == 0) {
        B->tuned = false;
        B->cluster = B->threads = 0;
    } else {
        if (cluster_ctas < 1 || cluster_ctas > 16 || (threads != 128 && threads != 256 && threads != 512))
            return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_set_shape: cluster 1..16, threads 128/256/512");
        const int minb = std::max(1, env_int("CUFSP_BATCH_MINB", 1));
        std::string why;
        auto k = batch_kernel(shape_source(B, threads, minb), why);
        if (!k) return set_error(CUFSP_ERR_CUDA, "cufsp_batch_set_shape: " + why);
        const int ncl = clusters_for(B, *k, cluster_ctas, threads);
        if (ncl < 1) return set_error(CUFSP_ERR_UNSUPPORTED, "cufsp_batch_set_shape: shape does not fit the device");
        cufsp_status s = ensure_work(B, ncl);
        if (s != CUFSP_SUCCESS) return s;
        B->cluster = cluster_ctas;
        B->threads = threads;
        B->minb = minb;
        B->kern = k;
        B->n_clusters = ncl;
        B->tuned = true;
        B->describe = describe_shape(B);
    }
    if (B->gexec) {
        cudaGraphExecDestroy(B->gexec);
        B->gexec = nullptr;
    }
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_batch_solve(cufsp_batch *B, double t_final, double *d_packed, cufsp_stream_t stream,
                                          cufsp_batch_stat *stats) {
    if (!B || !d_packed) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_solve: NULL argument");
    if (!(t_final >= 0.0) || !std::isfinite(t_final)) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_solve: bad t_final");
    cudaStream_t st = (cudaStream_t)stream;
    if (!B->tuned) {
        cufsp_status s = autotune(B, t_final, d_packed, st);
        if (s != CUFSP_SUCCESS) return s;
        if (B->gexec) {
            cudaGraphExecDestroy(B->gexec);
            B->gexec = nullptr;
        }
    }
    // replay the solve as a CUDA graph (re-captured when the final time, the vectors or the stream change)
    if (!B->gexec || B->g_tfinal != t_final || B->g_p != d_packed || B->g_stream != st) {
        if (B->gexec) {
            cudaGraphExecDestroy(B->gexec);
            B->gexec = nullptr;
        }
        cudaStream_t cs;
        CUFSP_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t g;
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        cufsp_status s = CUFSP_SUCCESS;
        if (e == cudaSuccess)
            s = launch(B, *B->kern, B->cluster, B->threads, B->n_clusters, t_final, d_packed, B->d_order, B->n_inst, cs);
        cudaError_t e2 = cudaStreamEndCapture(cs, &g);
        cudaStreamDestroy(cs);
        if (e != cudaSuccess || s != CUFSP_SUCCESS || e2 != cudaSuccess) {
            cudaGetLastError();
            return s != CUFSP_SUCCESS ? s : set_error(CUFSP_ERR_CUDA, "cufsp_batch_solve: graph capture failed");
        }
        e = cudaGraphInstantiate(&B->gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_error(e, "cufsp_batch_solve: graph instantiate");
        B->g_tfinal = t_final;
        B->g_p = d_packed;
        B->g_stream = st;
    }
    CUFSP_CUDA_TRY(cudaGraphLaunch(B->gexec, st));
    std::vector<CufspBatchStat> hs(B->n_inst);
    CUFSP_CUDA_TRY(cudaMemcpyAsync(hs.data(), B->d_stats, sizeof(CufspBatchStat) * B->n_inst, cudaMemcpyDeviceToHost, st));
    CUFSP_CUDA_TRY(cudaStreamSynchronize(st));
    cufsp_status ret = CUFSP_SUCCESS;
    for (int i = 0; i < B->n_inst; ++i) {
        if (stats) {
            stats[i].t = hs[i].t;
            stats[i].err = hs[i].err;
            stats[i].steps = hs[i].steps;
            stats[i].rejects = hs[i].rejects;
            stats[i].matvecs = hs[i].matvecs;
            stats[i].status = hs[i].status;
        }
        if (ret == CUFSP_SUCCESS && hs[i].status == 1) ret = set_error(CUFSP_ERR_STEP_LIMIT, "batched solve: an instance hit its step limit");
        if (ret == CUFSP_SUCCESS && hs[i].status == 2) ret = set_error(CUFSP_ERR_NONFINITE, "batched solve: NaN/Inf in an instance");
    }
    return ret;
}

extern "C" cufsp_status cufsp_batch_describe(const cufsp_batch *B, char *buf, size_t len) {
    if (!B || !buf || len == 0) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_batch_describe: bad argument");
    const std::string d = B->describe.empty() ? std::string("batched Krylov (launch shape not chosen yet)") : B->describe;
    const size_t k = std::min(len - 1, d.size());
    std::memcpy(buf, d.data(), k);
    buf[k] = 0;
    return CUFSP_SUCCESS;
}
