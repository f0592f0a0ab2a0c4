// cufsp_mat.cu -- the generator object behind the C ABI (replaces cuFSP::FSPMat,
// src/FSPMat.h:21-56, src/FSPMat.cu:10-118).
#include <algorithm>
#include <cmath>
#include <cstring>

#include <cstdlib>

#include "cufsp_internal.h"

using namespace cufsp;

namespace cufsp {

cufsp_status mat_coefs(cufsp_mat *A, double t, const double *coefs_in, std::vector<double> &out) {
    const int nr = A->model.nr;
    out.assign(nr, 1.0);
    if (coefs_in) {
        std::copy(coefs_in, coefs_in + nr, out.begin());
    } else if (A->model.tcoef) {
        A->model.tcoef(t, out.data(), A->model.tcoef_user);  // FSPMat::action: tcoeffunc(t, tcoef)
    }
    for (double c : out)
        if (!std::isfinite(c)) return set_error(CUFSP_ERR_NONFINITE, "time coefficient c_r(t) is NaN/Inf");
    return CUFSP_SUCCESS;
}

cufsp_status mat_apply(cufsp_mat *A, const double *coefs, double alpha, const double *d_alpha, const int *d_skip,
                       const double *x, bool accumulate, double *y, cudaStream_t st, int64_t i_begin, int64_t i_end) {
    if (A->kron) return kron_apply(A->kron, coefs, alpha, d_alpha, d_skip, x, accumulate, y, st, i_begin, i_end);
    return sparse_apply(A->sparse, coefs, alpha, d_alpha, d_skip, x, accumulate, y, st, i_begin, i_end);
}

cufsp_status mat_prepare(cufsp_mat *A, const double *coefs, cudaStream_t st, bool transpose) {
    return A->kron ? kron_prepare(A->kron, coefs, st, transpose) : CUFSP_SUCCESS;
}

cufsp_status mat_apply_transpose(cufsp_mat *A, const double *coefs, double alpha, const double *d_alpha,
                                 const int *d_skip, const double *x, double *y, cudaStream_t st) {
    if (!A->kron) return set_error(CUFSP_ERR_UNSUPPORTED, "transposed generator action needs the KRONECKER format");
    return kron_apply_transpose(A->kron, coefs, alpha, d_alpha, d_skip, x, y, st);
}

}  // namespace cufsp

extern "C" cufsp_status cufsp_mat_create(const cufsp_model_desc *desc, cufsp_format format, cufsp_mat **out) {
    clear_error();
    if (!out) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_create: out is NULL");
    *out = nullptr;
    if (format != CUFSP_FORMAT_CSR && format != CUFSP_FORMAT_HYB && format != CUFSP_FORMAT_KRONECKER)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_create: requested format is not supported");
    cufsp_mat *A = new cufsp_mat();
    A->format = format;
    cufsp_status s = model_from_desc(desc, format == CUFSP_FORMAT_KRONECKER, A->model);
    if (s == CUFSP_SUCCESS) {
        int dev_count = 0;
        cudaError_t e = cudaGetDeviceCount(&dev_count);
        if (e != cudaSuccess || dev_count == 0) s = set_error(CUFSP_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (s == CUFSP_SUCCESS) {
        if (format == CUFSP_FORMAT_KRONECKER) s = kron_create(A->model, &A->kron);
        else s = sparse_create(A->model, &A->sparse);
    }
    if (s != CUFSP_SUCCESS) {
        cufsp_mat_destroy(A);
        return s;
    }
    *out = A;
    return CUFSP_SUCCESS;
}

// Sparse-format generator from propensities the caller evaluated on the host, for models whose
// propensity is host code (the legacy cme::Model::propensity, src/Model.h:14-26) rather than a device
// PropFun or factor tables: prop_table[r * n + i] = a_r(x_i), n = number of states.
extern "C" cufsp_status cufsp_mat_create_table(const cufsp_model_desc *desc, cufsp_format format,
                                               const double *prop_table, cufsp_mat **out) {
    clear_error();
    if (!out || !desc || !prop_table) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_create_table: NULL argument");
    *out = nullptr;
    if (format != CUFSP_FORMAT_CSR && format != CUFSP_FORMAT_HYB)
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_create_table: a propensity table makes a CSR or HYB generator");
    cufsp_model_desc d = *desc;  // the table is the propensity source: the descriptor's own are ignored
    d.factor_tables = nullptr;
    d.prop_factor = nullptr;
    d.prop_device = nullptr;
    cufsp_mat *A = new cufsp_mat();
    A->format = format;
    cufsp_status s = model_from_desc(&d, false, A->model, /*external_table=*/true);
    if (s == CUFSP_SUCCESS) {
        const size_t cnt = (size_t)A->model.nr * (size_t)A->model.n;
        A->model.prop_table.assign(prop_table, prop_table + cnt);
        for (double v : A->model.prop_table)
            if (!std::isfinite(v)) {
                s = set_error(CUFSP_ERR_NONFINITE, "cufsp_mat_create_table: propensity table holds NaN/Inf");
                break;
            }
    }
    if (s == CUFSP_SUCCESS) {
        int dev_count = 0;
        const cudaError_t e = cudaGetDeviceCount(&dev_count);
        if (e != cudaSuccess || dev_count == 0) s = set_error(CUFSP_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (s == CUFSP_SUCCESS) s = sparse_create(A->model, &A->sparse);
    A->model.prop_table.clear();
    A->model.prop_table.shrink_to_fit();
    if (s != CUFSP_SUCCESS) {
        cufsp_mat_destroy(A);
        return s;
    }
    *out = A;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_mat_destroy(cufsp_mat *A) {
    if (!A) return CUFSP_SUCCESS;
    if (A->kron) kron_destroy(A->kron);
    if (A->sparse) sparse_destroy(A->sparse);
    if (A->d_x) cudaFree(A->d_x);
    if (A->d_y) cudaFree(A->d_y);
    for (cudaEvent_t e : A->ev) cudaEventDestroy(e);
    if (A->s_in) cudaStreamDestroy(A->s_in);
    if (A->s_comp) cudaStreamDestroy(A->s_comp);
    if (A->s_out) cudaStreamDestroy(A->s_out);
    delete A;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_mat_num_states(const cufsp_mat *A, int64_t *n) {
    if (!A || !n) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_num_states: bad argument");
    *n = A->model.n;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_mat_dims(const cufsp_mat *A, int *ns, int *nr, cufsp_format *format) {
    if (!A) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_dims: A is NULL");
    if (ns) *ns = A->model.ns;
    if (nr) *nr = A->model.nr;
    if (format) *format = A->format;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_mat_apply(cufsp_mat *A, double t, const double *coefs, double alpha, const double *x,
                                        double beta, double *y, cufsp_stream_t stream) {
    if (!A || !x || !y) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_apply: NULL argument");
    if (beta != 0.0 && beta != 1.0) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_apply: beta must be 0 or 1");
    if (x == y) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_apply: x and y must not alias");
    if (!std::isfinite(alpha)) return set_error(CUFSP_ERR_NONFINITE, "cufsp_mat_apply: alpha is NaN/Inf");
    cufsp_status s = mat_coefs(A, t, coefs, A->coef_buf);
    if (s != CUFSP_SUCCESS) return s;
    return mat_apply(A, A->coef_buf.data(), alpha, nullptr, nullptr, x, beta != 0.0, y, (cudaStream_t)stream);
}

extern "C" cufsp_status cufsp_mat_apply_transpose(cufsp_mat *A, double t, const double *coefs, double alpha,
                                                  const double *x, double *y, cufsp_stream_t stream) {
    if (!A || !x || !y) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_apply_transpose: NULL argument");
    if (x == y) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_apply_transpose: x and y must not alias");
    if (!std::isfinite(alpha)) return set_error(CUFSP_ERR_NONFINITE, "cufsp_mat_apply_transpose: alpha is NaN/Inf");
    cufsp_status s = mat_coefs(A, t, coefs, A->coef_buf);
    if (s != CUFSP_SUCCESS) return s;
    return mat_apply_transpose(A, A->coef_buf.data(), alpha, nullptr, nullptr, x, y, (cudaStream_t)stream);
}

extern "C" cufsp_status cufsp_mat_action(cufsp_mat *A, double t, const double *x, double *y, cufsp_stream_t stream) {
    return cufsp_mat_apply(A, t, nullptr, 1.0, x, 1.0, y, stream);
}

extern "C" cufsp_status cufsp_mat_watchdog(cufsp_mat *A, int *tripped) {
    if (!A || !tripped) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_watchdog: NULL argument");
    CUFSP_CUDA_TRY(cudaDeviceSynchronize());  // every launch of the generator has finished
    *tripped = A->kron ? kron_watchdog(A->kron) : 0;
    return CUFSP_SUCCESS;
}

namespace cufsp {
cufsp_status mat_check_watchdog(cufsp_mat *A, const char *where) {
    if (A && A->kron && kron_watchdog(A->kron))
        return set_error(CUFSP_ERR_CUDA, std::string(where) +
                                             ": a bounded shared-memory barrier wait of the generator kernel expired "
                                             "(the generator action is incomplete)");
    return CUFSP_SUCCESS;
}
}  // namespace cufsp

extern "C" cufsp_status cufsp_mat_describe(const cufsp_mat *A, char *buf, size_t len) {
    if (!A || !buf || len == 0) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_describe: bad argument");
    const std::string d = A->kron ? "KRONECKER: " + kron_describe(A->kron) : sparse_describe(A->sparse);
    const size_t k = std::min(len - 1, d.size());
    std::memcpy(buf, d.data(), k);
    buf[k] = 0;
    return CUFSP_SUCCESS;
}

extern "C" cufsp_status cufsp_mat_export_propensities(const cufsp_mat *A, double *d_props, cufsp_stream_t stream) {
    if (!A || !d_props) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_export_propensities: NULL argument");
    if (!A->sparse) return set_error(CUFSP_ERR_UNSUPPORTED, "propensity export needs the CSR/HYB format");
    return sparse_export(A->sparse, d_props, (cudaStream_t)stream);
}

// Host-buffer action: slabs of whole rows stream in on s_in, are applied on s_comp as soon as
// their x halo has arrived, and stream back on s_out, so H2D, compute and D2H overlap.
extern "C" cufsp_status cufsp_mat_action_host(cufsp_mat *A, double t, const double *x_host, double *y_host) {
    if (!A || !x_host || !y_host) return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_mat_action_host: NULL argument");
    cufsp_status s = mat_coefs(A, t, nullptr, A->coef_buf);
    if (s != CUFSP_SUCCESS) return s;
    const int64_t n = A->model.n;
    // Slabs of whole rows/planes (CUFSP_HOST_SLABS overrides the 8, 1..64): on the 255^3 workload 8
    // slabs moved 71.5 GB/s of y += A x through PCIe, 16 slabs 70.3 and 32 slabs 65.8.
    static const int kSlabs = [] {
        const char *e = getenv("CUFSP_HOST_SLABS");
        const int v = e ? atoi(e) : 8;
        return v < 1 ? 1 : (v > 64 ? 64 : v);
    }();
    if (!A->d_x) {
        CUFSP_CUDA_TRY(dev_malloc(&A->d_x, sizeof(double) * n));
        CUFSP_CUDA_TRY(dev_malloc(&A->d_y, sizeof(double) * n));
        CUFSP_CUDA_TRY(cudaStreamCreateWithFlags(&A->s_in, cudaStreamNonBlocking));
        CUFSP_CUDA_TRY(cudaStreamCreateWithFlags(&A->s_comp, cudaStreamNonBlocking));
        CUFSP_CUDA_TRY(cudaStreamCreateWithFlags(&A->s_out, cudaStreamNonBlocking));
        A->ev.resize(3 * kSlabs);
        for (auto &e : A->ev) CUFSP_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    const int64_t gran = A->kron ? kron_row_len(A->kron) : 1;
    const int64_t halo = A->kron ? kron_halo(A->kron) : sparse_halo(A->sparse);
    const int64_t rows = n / gran;
    std::vector<int64_t> b(kSlabs + 1);
    for (int k = 0; k <= kSlabs; ++k) b[k] = (rows * k / kSlabs) * gran;
    cudaEvent_t *evx = A->ev.data(), *evy = evx + kSlabs, *evc = evy + kSlabs;
    // One host->device stream: a second one for the y slabs moved the same 71 GB/s (the PCIe link).
    cudaStream_t ys = A->s_in;
    for (int k = 0; k < kSlabs; ++k) {
        const int64_t cnt = b[k + 1] - b[k];
        if (cnt > 0) {
            CUFSP_CUDA_TRY(cudaMemcpyAsync(A->d_x + b[k], x_host + b[k], sizeof(double) * cnt, cudaMemcpyHostToDevice, A->s_in));
        }
        CUFSP_CUDA_TRY(cudaEventRecord(evx[k], A->s_in));
        if (cnt > 0) {
            CUFSP_CUDA_TRY(cudaMemcpyAsync(A->d_y + b[k], y_host + b[k], sizeof(double) * cnt, cudaMemcpyHostToDevice, ys));
        }
        CUFSP_CUDA_TRY(cudaEventRecord(evy[k], ys));
    }
    for (int k = 0; k < kSlabs; ++k) {
        const int64_t cnt = b[k + 1] - b[k];
        if (cnt <= 0) continue;
        // last slab whose x is needed: the one holding index b[k+1] - 1 + halo
        const int64_t need = std::min<int64_t>(n - 1, b[k + 1] - 1 + halo);
        int kk = k;
        while (kk + 1 < kSlabs && b[kk + 1] <= need) ++kk;
        CUFSP_CUDA_TRY(cudaStreamWaitEvent(A->s_comp, evx[kk], 0));
        CUFSP_CUDA_TRY(cudaStreamWaitEvent(A->s_comp, evy[k], 0));
        s = mat_apply(A, A->coef_buf.data(), 1.0, nullptr, nullptr, A->d_x, true, A->d_y, A->s_comp, b[k], b[k + 1]);
        if (s != CUFSP_SUCCESS) return s;
        CUFSP_CUDA_TRY(cudaEventRecord(evc[k], A->s_comp));
        CUFSP_CUDA_TRY(cudaStreamWaitEvent(A->s_out, evc[k], 0));
        CUFSP_CUDA_TRY(cudaMemcpyAsync(y_host + b[k], A->d_y + b[k], sizeof(double) * cnt, cudaMemcpyDeviceToHost, A->s_out));
    }
    CUFSP_CUDA_TRY(cudaStreamSynchronize(A->s_out));
    CUFSP_CUDA_TRY(cudaStreamSynchronize(A->s_comp));
    return mat_check_watchdog(A, "cufsp_mat_action_host");
}
