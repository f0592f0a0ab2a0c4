// ref_shim.cu -- C entry points into the reference's OWN compiled sources (TEST INFRASTRUCTURE).
//
// Built by oracle/Makefile (target `ref`) together with the unmodified reference files
// src/cme_util.cu, src/fspmat_hyb_kernels.cu and src/fspmat_kron_kernels.cu of voduchuy/CUDA_FSP,
// read in place at build time.  The output goes to oracle/_ref/ and is used only by tests/ to pin
// the oracle and the product against the reference's own arithmetic:
//   host:  rect_fsp_num_states, indx2state, state2indx (src/cme_util.cu:5-22,55-62),
//          fspmat_sdkron_fill_host_data (src/fspmat_kron_kernels.cu:170-190)
//   GPU:   fsp_get_states (src/cme_util.cu:24-41), the HYB build + action
//          (src/fspmat_hyb_kernels.cu:66-184) with the toggle PropFun or a factor-table PropFun, and
//          the Kronecker action (src/fspmat_kron_kernels.cu:31-168); both actions also timed.
// The GPU entry points are only called with state counts that are multiples of 1024: the HYB action
// has a __syncthreads() inside `if (tid < n_states)` (fspmat_hyb_kernels.cu:71-76) and the Kronecker
// grid drops the last partial block (fspmat_kron_kernels.cu:42), so other sizes are not run.
#include <cstdio>
#include <cstring>
#include <vector>

#include "cme_util.h"
#include "fspmat_hyb_kernels.h"
#include "fspmat_kron_kernels.h"

// The two-gene toggle switch propensity of the reference tests (tests/test_fsp_mat.cu:19-50).
namespace {
const double kAyx = 2.6e-3, kAxy = 6.1e-3, kNyx = 3e0, kNxy = 2.1e0;
}

__device__ double shim_toggle_propensity(int *x, int reaction) {
    switch (reaction) {
        case 0: return 1.0;
        case 1: return 1.0 / (1.0 + kAyx * pow(1.0 * x[1], kNyx));
        case 2: return 1.0 * x[0];
        case 3: return 1.0;
        case 4: return 1.0 / (1.0 + kAxy * pow(1.0 * x[0], kNxy));
        case 5: return 1.0 * x[1];
        default: return 0.0;
    }
}
__device__ cuFSP::PropFun shim_toggle_ptr = &shim_toggle_propensity;

// A factor-table propensity a_r(x) = prod_s f_{r,s}(x_s) as a device PropFun, for running the
// reference's HYB format on the product's factorised workloads (tables set by set_device_tables).
__device__ const double *shim_dev_tables;
__device__ int shim_dev_off[16];
__device__ int shim_dev_stride;
__device__ int shim_dev_ns;

__device__ double shim_table_propensity(int *x, int reaction) {
    const double *t = shim_dev_tables + (size_t)reaction * shim_dev_stride;
    double v = 1.0;
    for (int s = 0; s < shim_dev_ns; ++s) v *= t[shim_dev_off[s] + x[s]];
    return v;
}
__device__ cuFSP::PropFun shim_table_ptr = &shim_table_propensity;

// Copies the factor tables to the device for shim_table_propensity; returns the device copy.
static double *set_device_tables(int ns, int nr, const int *bounds, const double *tables) {
    int off[16] = {0};
    int stride = 0;
    for (int s = 0; s < ns && s < 16; ++s) {
        off[s] = stride;
        stride += bounds[s] + 1;
    }
    double *d_tab = nullptr;
    cudaMalloc(&d_tab, sizeof(double) * (size_t)nr * stride);
    cudaMemcpy(d_tab, tables, sizeof(double) * (size_t)nr * stride, cudaMemcpyHostToDevice);
    cudaMemcpyToSymbol(shim_dev_tables, &d_tab, sizeof(d_tab));
    cudaMemcpyToSymbol(shim_dev_off, off, sizeof(off));
    cudaMemcpyToSymbol(shim_dev_stride, &stride, sizeof(int));
    cudaMemcpyToSymbol(shim_dev_ns, &ns, sizeof(int));
    return d_tab;
}

static const double *g_tables = nullptr;
static std::vector<int> g_off;
static int g_stride = 0;

static double shim_table_factor(int x, int species, int reaction) {
    return g_tables[(size_t)reaction * g_stride + g_off[species] + x];
}

static void set_tables(int ns, const int *bounds, const double *tables) {
    g_tables = tables;
    g_off.assign(ns, 0);
    int off = 0;
    for (int s = 0; s < ns; ++s) {
        g_off[s] = off;
        off += bounds[s] + 1;
    }
    g_stride = off;
}

static cuFSP::CSRMatInt make_stoich(int nr, int ns, int *sv, int *sc, int *sr) {
    cuFSP::CSRMatInt st;
    st.vals = sv;
    st.col_idxs = sc;
    st.row_ptrs = sr;
    st.n_rows = nr;
    st.n_cols = ns;
    st.nnz = sr[nr];
    return st;
}

extern "C" {

int ref_num_states(int ns, int *bounds) { return cuFSP::rect_fsp_num_states(ns, bounds); }

void ref_indx2state(int indx, int *state, int ns, int *bounds) { cuFSP::indx2state(indx, state, ns, bounds); }

int ref_state2indx(int *state, int ns, int *bounds) { return cuFSP::state2indx(state, ns, bounds); }

// vals_out: nr * sum(b+1) doubles; offsets_out: nr * ns ints.
void ref_sdkron_fill(int ns, int *bounds, int nr, int *sv, int *sc, int *sr, const double *tables,
                     double *vals_out, int *offsets_out) {
    set_tables(ns, bounds, tables);
    cuFSP::fspmat_sdkron_fill_host_data(ns, bounds, nr, make_stoich(nr, ns, sv, sc, sr), &shim_table_factor,
                                        vals_out, offsets_out);
}

// ---- GPU entry points (run on a CUDA device only) ----

int ref_gpu_get_states(int ns, int *bounds, int *states_host) {
    int n = cuFSP::rect_fsp_num_states(ns, bounds);
    int *d_b = nullptr, *d_s = nullptr;
    cudaMalloc(&d_b, ns * sizeof(int));
    cudaMalloc(&d_s, (size_t)n * ns * sizeof(int));
    cudaMemcpy(d_b, bounds, ns * sizeof(int), cudaMemcpyHostToDevice);
    int blocks = (n + 1023) / 1024;
    cuFSP::fsp_get_states<<<blocks, 1024, ns * sizeof(int)>>>(d_s, ns, n, d_b);
    cudaError_t e = cudaDeviceSynchronize();
    cudaMemcpy(states_host, d_s, (size_t)n * ns * sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d_b);
    cudaFree(d_s);
    return (int)e;
}

// y_host += sum_r coefs[r] A_r x_host with the reference HYB format and the toggle propensity.
int ref_gpu_hyb_toggle(int *bounds, const double *coefs, const double *x_host, double *y_host) {
    int sv[] = {1, 1, -1, 1, 1, -1}, sc[] = {0, 0, 0, 1, 1, 1}, sr[] = {0, 1, 2, 3, 4, 5, 6};
    int n = cuFSP::rect_fsp_num_states(2, bounds);
    if (n % 1024 != 0) return -1;
    cuFSP::PropFun prop = nullptr;
    cudaMemcpyFromSymbol(&prop, shim_toggle_ptr, sizeof(cuFSP::PropFun));
    cuFSP::HYBMatSet hyb;
    cuFSP::generate_fsp_mats_hyb(n, 6, 2, bounds, make_stoich(6, 2, sv, sc, sr), prop, &hyb);
    double *d_x = nullptr, *d_y = nullptr;
    cudaMalloc(&d_x, n * sizeof(double));
    cudaMalloc(&d_y, n * sizeof(double));
    cudaMemcpy(d_x, x_host, n * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(d_y, y_host, n * sizeof(double), cudaMemcpyHostToDevice);
    std::vector<double> c(coefs, coefs + 6);
    hyb.action(d_x, d_y, c.data());
    cudaError_t e = cudaMemcpy(y_host, d_y, n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_x);
    cudaFree(d_y);
    hyb.destroy();
    return (int)e;
}

// y_host += sum_r coefs[r] A_r x_host with the reference Kronecker format built from `tables`.
int ref_gpu_kron(int ns, int nr, int *bounds, int *sv, int *sc, int *sr, const double *tables, const double *coefs,
                 const double *x_host, double *y_host) {
    int n = cuFSP::rect_fsp_num_states(ns, bounds);
    if (n % 1024 != 0) return -1;
    set_tables(ns, bounds, tables);
    cuFSP::SDKronMatSet kr;
    cuFSP::generate_fsp_mats_sdkron(nr, ns, bounds, make_stoich(nr, ns, sv, sc, sr), &shim_table_factor, &kr);
    double *d_x = nullptr, *d_y = nullptr;
    cudaMalloc(&d_x, (size_t)n * sizeof(double));
    cudaMalloc(&d_y, (size_t)n * sizeof(double));
    cudaMemcpy(d_x, x_host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(d_y, y_host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    std::vector<double> c(coefs, coefs + nr);
    kr.action(d_x, d_y, c.data());
    cudaError_t e = cudaMemcpy(y_host, d_y, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_x);
    cudaFree(d_y);
    kr.destroy();
    return (int)e;
}

// The reference HYB format built through its own fill kernel with the factor-table PropFun above.
// With x_host / y_host: y_host += sum_r coefs[r] A_r x_host (returns a CUDA error code).  With
// iters > 0 and null vectors: `iters` actions on device buffers timed with cudaEvent, ms per action
// returned through *ms.
int ref_gpu_hyb_tables(int ns, int nr, int *bounds, int *sv, int *sc, int *sr, const double *tables,
                       const double *coefs, const double *x_host, double *y_host, int iters, double *ms) {
    int n = cuFSP::rect_fsp_num_states(ns, bounds);
    if (n % 1024 != 0) return -1;
    double *d_tab = set_device_tables(ns, nr, bounds, tables);
    cuFSP::PropFun prop = nullptr;
    cudaMemcpyFromSymbol(&prop, shim_table_ptr, sizeof(cuFSP::PropFun));
    cuFSP::HYBMatSet hyb;
    cuFSP::generate_fsp_mats_hyb(n, nr, ns, bounds, make_stoich(nr, ns, sv, sc, sr), prop, &hyb);
    double *d_x = nullptr, *d_y = nullptr;
    cudaMalloc(&d_x, (size_t)n * sizeof(double));
    cudaMalloc(&d_y, (size_t)n * sizeof(double));
    std::vector<double> c(coefs, coefs + nr);
    cudaError_t e = cudaSuccess;
    if (x_host && y_host) {
        cudaMemcpy(d_x, x_host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
        cudaMemcpy(d_y, y_host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
        hyb.action(d_x, d_y, c.data());
        e = cudaMemcpy(y_host, d_y, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    } else if (iters > 0 && ms) {
        cudaMemset(d_x, 0, (size_t)n * sizeof(double));
        cudaMemset(d_y, 0, (size_t)n * sizeof(double));
        hyb.action(d_x, d_y, c.data());
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a);
        for (int i = 0; i < iters; ++i) hyb.action(d_x, d_y, c.data());
        cudaEventRecord(b);
        e = cudaEventSynchronize(b);
        float t = 0.f;
        cudaEventElapsedTime(&t, a, b);
        *ms = t / iters;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    cudaFree(d_x);
    cudaFree(d_y);
    cudaFree(d_tab);
    hyb.destroy();
    return (int)e;
}

// Time `iters` Kronecker actions on device buffers (cudaEvent); returns ms per action.
double ref_gpu_kron_time(int ns, int nr, int *bounds, int *sv, int *sc, int *sr, const double *tables,
                         const double *coefs, int iters) {
    int n = cuFSP::rect_fsp_num_states(ns, bounds);
    if (n % 1024 != 0) return -1.0;
    set_tables(ns, bounds, tables);
    cuFSP::SDKronMatSet kr;
    cuFSP::generate_fsp_mats_sdkron(nr, ns, bounds, make_stoich(nr, ns, sv, sc, sr), &shim_table_factor, &kr);
    double *d_x = nullptr, *d_y = nullptr;
    cudaMalloc(&d_x, (size_t)n * sizeof(double));
    cudaMalloc(&d_y, (size_t)n * sizeof(double));
    cudaMemset(d_x, 0, (size_t)n * sizeof(double));
    cudaMemset(d_y, 0, (size_t)n * sizeof(double));
    std::vector<double> c(coefs, coefs + nr);
    kr.action(d_x, d_y, c.data());
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a);
    for (int i = 0; i < iters; ++i) kr.action(d_x, d_y, c.data());
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaFree(d_x);
    cudaFree(d_y);
    kr.destroy();
    return ms / iters;
}
}
