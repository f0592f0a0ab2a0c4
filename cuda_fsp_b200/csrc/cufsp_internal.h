// cufsp_internal.h -- shared declarations of the cufsp CUDA library (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <string>
#include <vector>

#include "../../include/cufsp.h"

#define CUFSP_MAX_SPECIES 16
#define CUFSP_MAX_REACTIONS 32   // KRONECKER register path; the sparse path allows CUFSP_MAX_REACTIONS_SPARSE
#define CUFSP_MAX_REACTIONS_SPARSE 256
#define CUFSP_MAX_KRYLOV 60  // m + 1 basis vectors must fit the 64-wide multi-vector kernels

namespace cufsp {

// Thread-local last-error text; set_error returns the status for `return set_error(...)`.
cufsp_status set_error(cufsp_status s, const std::string &msg);
cufsp_status cuda_error(cudaError_t e, const char *what);
void clear_error();

#define CUFSP_CUDA_TRY(call)                                              \
    do {                                                                  \
        cudaError_t _e = (call);                                          \
        if (_e != cudaSuccess) return ::cufsp::cuda_error(_e, #call);     \
    } while (0)

// Device properties cached per device id.
struct DeviceInfo {
    int sm_count = 0;
    int max_smem_optin = 0;
};
const DeviceInfo &device_info();

// Fast unsigned division by a runtime constant for numerators < 2^31
// (round-up multiplier method of Granlund & Montgomery, PLDI 1994):
//   l = ceil(log2 d), M = floor(2^32 (2^l - d) / d) + 1, q = (umulhi(M, n) + n) >> l.
struct FastDiv {
    uint32_t d;
    uint32_t mul;
    uint32_t shift;
};
FastDiv make_fastdiv(uint32_t d);

#if defined(__CUDACC__)
__host__ __device__ __forceinline__ uint32_t fd_div(uint32_t n, const FastDiv &f) {
#if defined(__CUDA_ARCH__)
    uint32_t t = __umulhi(n, f.mul);
#else
    uint32_t t = (uint32_t)(((uint64_t)n * f.mul) >> 32);
#endif
    return (t + n) >> f.shift;
}
#endif

// Device buffers from a per-process cache (cufsp_common.cu).  cache_free(p, st): every use of p was
// ordered on stream st; the buffer is kept and its next owner waits for st to reach this point.
// cache_free(p): uses unknown; synchronises p's device first.  dev_malloc: cudaMalloc that returns
// the cache's idle buffers of the current device to the driver and retries when memory runs out.
cudaError_t cache_alloc(void **p, size_t bytes);
void cache_free(void *p);
void cache_free(void *p, cudaStream_t last_use);
cudaError_t dev_malloc(void **p, size_t bytes);
size_t cache_trim_all();
// cudaMemcpy from pageable memory returns once the data is staged, and cudaMemset once it is
// queued, both on the legacy default stream, which streams created non-blocking (the batched
// gradient's workers, the host-buffer action) do not wait for.  Uploads of data that such streams
// read end with upload_fence(): it returns when the legacy stream's queued work has finished.
cudaError_t upload_fence();
// One pinned host double from pages that stay allocated for the process: cudaHostAlloc and
// cudaFreeHost synchronise the device, which would stall concurrent solves on other streams every
// time a Krylov driver is created or destroyed.  Null when pinned memory is exhausted.
double *pinned_slot_get();
void pinned_slot_put(double *p);
template <class T>
cudaError_t dev_malloc(T **p, size_t bytes) {
    return dev_malloc(reinterpret_cast<void **>(p), bytes);
}

// Watchdog word of a kernel with bounded waits: pinned host memory mapped into the device, so the
// host reads it after any synchronisation of the launching stream without another copy.
// Returns the host address (0 written) and the device address in *d_word; nullptr on failure.
int *watch_word_alloc(int **d_word);
void watch_word_free(int *h_word);
// Reads and clears a watchdog word (the caller has synchronised the stream of the kernels using it).
int watch_word_take(int *h_word);

// Reduction scratch shared by the vector kernels of one handle: per-CTA partials and a
// completion counter for the last-CTA-reduces pattern (deterministic summation order).
struct ReduceScratch {
    double *partials = nullptr;  // [max_ctas * max_k]
    unsigned int *counter = nullptr;
    int max_ctas = 0;
    int max_k = 0;
    cufsp_status init(int max_ctas, int max_k);                   // counter zeroed before return
    cufsp_status init(int max_ctas, int max_k, cudaStream_t st);  // counter zeroed in order on st
    void release();
    void release(cudaStream_t last_use);
};

// Grid for a streaming vector kernel of n elements with 256 threads per CTA.
int stream_grid(int64_t n, int elems_per_thread, int max_ctas);

// sum / dot / norm primitives (cufsp_common.cu)
cufsp_status launch_sum(int64_t n, const double *x, double *d_out, ReduceScratch &rs, cudaStream_t st);
cufsp_status launch_nrm2(int64_t n, const double *x, double *d_out, ReduceScratch &rs, cudaStream_t st);
cufsp_status launch_fill(int64_t n, double *x, double v, cudaStream_t st);
cufsp_status launch_scale(int64_t n, double *x, const double *d_alpha, double alpha, cudaStream_t st);

// Model data validated and normalised on the host.
struct ModelHost {
    int ns = 0, nr = 0;
    int64_t n = 0;
    std::vector<int> bounds;       // b_s
    std::vector<int> nu;           // dense stoichiometry [nr][ns]
    std::vector<double> tables;    // [nr][sum_s(b_s+1)] or empty
    std::vector<double> prop_table;  // [nr][n] propensities evaluated by the caller (sparse formats) or empty
    std::vector<int> tab_off;      // [ns] offset of species s inside a reaction's block
    int tab_stride = 0;            // sum_s (b_s + 1)
    cufsp_prop_fn prop_device = nullptr;
    cufsp_tcoef_fn tcoef = nullptr;
    void *tcoef_user = nullptr;
};
// external_table: the propensities come from a caller-evaluated table (cufsp_mat_create_table).
cufsp_status model_from_desc(const cufsp_model_desc *d, bool need_tables, ModelHost &m, bool external_table = false);

// ---- format back-ends ----------------------------------------------------------------------
struct KronData;    // matrix-free factorised generator (cufsp_kron.cu)
struct SparseData;  // reaction-major propensity table (cufsp_sparse.cu)

cufsp_status kron_create(const ModelHost &m, KronData **out);
void kron_destroy(KronData *k);
// y = alpha * A(coefs) x (+ y if accumulate); d_alpha (nullable) multiplies alpha on the device;
// the kernel returns at once when d_skip is non-null and *d_skip != 0.
// Rows [q_begin, q_end) of the outer index only (q_end < 0: all rows).
cufsp_status kron_apply(KronData *k, const double *coefs, double alpha, const double *d_alpha,
                        const int *d_skip, const double *x, bool accumulate, double *y, cudaStream_t st,
                        int64_t i_begin = 0, int64_t i_end = -1);
// Watchdog of the TMA-fed kernels: 1 if a bounded barrier wait expired since the last call (reset).
// Does not synchronise: the caller has synchronised the streams the generator's kernels ran on.
int kron_watchdog(KronData *k);
// halo (max |shift|) and slab granularity for the host-buffer pipeline
int64_t kron_halo(const KronData *k);
int64_t kron_row_len(const KronData *k);

cufsp_status sparse_create(const ModelHost &m, SparseData **out);
void sparse_destroy(SparseData *s);
cufsp_status sparse_apply(SparseData *s, const double *coefs, double alpha, const double *d_alpha,
                          const int *d_skip, const double *x, bool accumulate, double *y, cudaStream_t st,
                          int64_t i_begin = 0, int64_t i_end = -1);
cufsp_status sparse_export(const SparseData *s, double *d_props, cudaStream_t st);
int64_t sparse_halo(const SparseData *s);
const std::string &sparse_describe(const SparseData *s);

// Kernels compiled at run time by NVRTC for sm_100a (cufsp_rtc.cu): cached per process by source
// text; nullptr with the reason in `why` when compiling or loading fails.
struct RtcModule {
    cudaLibrary_t lib = nullptr;
    std::vector<cudaKernel_t> kernels;  // in the order of the requested names
    std::string log;
};
std::shared_ptr<RtcModule> rtc_module(const std::string &src, const std::vector<std::string> &names,
                                      std::string &why);

// Runtime-specialised plane kernel for near-neighbour networks of 2-3 species (cufsp_kron_plane.cu).
struct PlaneData;
// nullptr (with the reason in `why`) when the network does not have the plane kernel's shape or the
// kernel could not be compiled; d_tables: the generator's device factor tables.
PlaneData *plane_create(const ModelHost &m, const double *d_tables, std::string &why);
void plane_destroy(PlaneData *pd);
const std::string &plane_description(const PlaneData *pd);
int64_t plane_size(const PlaneData *pd);  // states per plane (slab granularity)
int plane_watchdog(PlaneData *pd);         // 1 if a bounded barrier wait expired since the last call (reset; no sync)
// false when this apply is not for the plane kernel (range not whole planes, unaligned vectors);
// otherwise launches and sets *status.
bool plane_launch(PlaneData *pd, const double *coefs, double alpha, const double *d_alpha, const int *d_skip,
                  const double *x, bool accumulate, double *y, cudaStream_t st, int64_t i_begin, int64_t i_end,
                  cufsp_status *status);
// Coefficient-dependent tables of the plane kernel (row words), rebuilt when the coefficients change.
cufsp_status plane_prepare(PlaneData *pd, const double *coefs, cudaStream_t st);
// transpose: the transposed action will follow (its kernel is compiled here, outside any capture).
cufsp_status kron_prepare(KronData *k, const double *coefs, cudaStream_t st, bool transpose = false);
// Human-readable kernel choice of a KRONECKER generator.
std::string kron_describe(const KronData *k);

// Transposed generator action y = alpha * A(coefs)^T x (overwrite), KRONECKER format
// (cufsp_adjoint.cu); d_alpha / d_skip as in kron_apply.
cufsp_status kron_apply_transpose(KronData *k, const double *coefs, double alpha, const double *d_alpha,
                                  const int *d_skip, const double *x, double *y, cudaStream_t st);

// Basis data of one Arnoldi pass (single-instance Krylov driver, cufsp_krylov.cu), for the adjoint.
struct KrylovStep {
    int mb = 0;               // basis size (m, or the happy-breakdown size)
    double beta = 0.0;        // ||v||
    double tau = 0.0;         // accepted step length (expv_step), 0 after a bare Arnoldi pass
    std::vector<double> H;    // leading mb x mb Hessenberg block, column-major
    std::vector<double> rho;  // v_k = rho_k W_k
};

// Host-side dense exponential (cufsp_expm.cpp).
cufsp_status expm_pade13(int k, const double *A, double *F);
// exp of [[A11, A12], [0, A22]] (k1 + k2 square, column-major; the lower-left block is not read)
cufsp_status expm_pade13_blocktri(int k1, int k2, const double *A, double *F);

}  // namespace cufsp

// Opaque handle behind cufsp_mat.
struct cufsp_mat_s {
    cufsp::ModelHost model;
    cufsp_format format = CUFSP_FORMAT_KRONECKER;
    cufsp::KronData *kron = nullptr;
    cufsp::SparseData *sparse = nullptr;
    std::vector<double> coef_buf;
    // host-buffer pipeline resources (created on first use)
    double *d_x = nullptr, *d_y = nullptr;
    cudaStream_t s_in = nullptr, s_comp = nullptr, s_out = nullptr;
    std::vector<cudaEvent_t> ev;
};

namespace cufsp {
// d_skip (nullable): the kernels return at once when *d_skip != 0 (Krylov breakdown / error flag).
cufsp_status mat_apply(cufsp_mat *A, const double *coefs, double alpha, const double *d_alpha, const int *d_skip,
                       const double *x, bool accumulate, double *y, cudaStream_t st, int64_t i_begin = 0,
                       int64_t i_end = -1);
cufsp_status mat_coefs(cufsp_mat *A, double t, const double *coefs_in, std::vector<double> &out);
// CUFSP_ERR_CUDA when one of the generator's kernels gave up a bounded wait since the last check
// (its output is then incomplete); called by the drivers after they synchronise their stream.
cufsp_status mat_check_watchdog(cufsp_mat *A, const char *where);
// Bring the generator's coefficient-dependent device tables up to `coefs` (stream order); applies
// captured in a CUDA graph after this call launch nothing else.
cufsp_status mat_prepare(cufsp_mat *A, const double *coefs, cudaStream_t st, bool transpose = false);
// y = alpha * A(coefs)^T x (overwrite); KRONECKER generators only.
cufsp_status mat_apply_transpose(cufsp_mat *A, const double *coefs, double alpha, const double *d_alpha,
                                 const int *d_skip, const double *x, double *y, cudaStream_t st);

// Persistent single-launch Arnoldi pass for generators whose Krylov basis stays in L2
// (cufsp_arnoldi.cu).  Writes the same device state block as the launch sequence of
// cufsp_krylov.cu; *err (zeroed here) is set when a bounded grid-barrier wait expired.
struct PArnoldi;
bool parnoldi_wanted(const cufsp_mat *A, int64_t n, int m);
bool parnoldi_size_ok(int64_t n);  // the size rule of parnoldi_wanted alone
cufsp_status parnoldi_run(PArnoldi **pa, cufsp_mat *A, const std::vector<double> &coefs, bool transpose,
                          int64_t n, const double *v, double *W, double *H, double *rho, double *gam, double *beta,
                          double *avnorm, int *flag, int *err, int m, int iop, int q, double btol, bool with_avnorm,
                          cudaStream_t st);
void parnoldi_destroy(PArnoldi *pa);
void parnoldi_destroy(PArnoldi *pa, cudaStream_t last_use);  // every launch of pa was ordered on last_use
// Host threads that run many solves concurrently keep the launch sequence: the persistent pass
// wants every SM to itself.
void parnoldi_thread_disable(bool off);
// Passes launched later from this host thread use at most `cap` CTAs (one per SM; 0: every SM), so
// that several threads' passes share the GPU side by side.
void parnoldi_thread_cta_cap(int cap);

// Internals of the single-instance Krylov driver used by the adjoint gradient (cufsp_krylov.cu).
void expv_set_transpose(cufsp_expv *E, bool transpose);
cufsp_status expv_arnoldi(cufsp_expv *E, double *v, cudaStream_t st);  // Arnoldi pass only
cufsp_status expv_step_once(cufsp_expv *E, double *v, cudaStream_t st);  // one accepted step
const KrylovStep &expv_last(const cufsp_expv *E);
const double *expv_basis(const cufsp_expv *E, const double *v, int k);  // W_k (W_0 = v)
}  // namespace cufsp
