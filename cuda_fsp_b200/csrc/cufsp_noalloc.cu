// cufsp_noalloc.cu -- vector sum that allocates no device memory (cufsp_vec_sum_noalloc).
//
// The reduction is the same deterministic two-level sum as cufsp_vec_sum (block partials, the last
// block to finish adds them in a fixed order), but its scratch -- one partial per block and the
// completion counter -- lives in a file-scope __device__ array instead of memory allocated per
// call.  The array is part of the library's device image: every GPU that loads the library holds
// it (8 KB) until the process exits.
#include <mutex>
#include <vector>

#include "cufsp_internal.h"
#include "cufsp_reduce.cuh"

namespace cufsp {
namespace {

constexpr int kNaBlocks = CUFSP_NOALLOC_MAX_N / 4096;  // one partial per 4096-element block
constexpr int kNaPerBlock = 4096;                      // 256 threads x 16 elements
static_assert((int64_t)kNaBlocks * kNaPerBlock == CUFSP_NOALLOC_MAX_N, "scratch sizing");

// [0, kNaBlocks): block partial sums; slot kNaBlocks: completion counter (unsigned int).
static __device__ __align__(256) double g_sum_scratch[kNaBlocks + 2];

__global__ void __launch_bounds__(kRedThreads) k_sum_noalloc(int64_t n, const double *__restrict__ x,
                                                            double *__restrict__ scratch, double *__restrict__ out) {
    __shared__ RedSmem<1> sm;
    double acc[1] = {0.0};
    const int64_t begin = (int64_t)blockIdx.x * kNaPerBlock;
    const int64_t end = begin + kNaPerBlock < n ? begin + kNaPerBlock : n;
    for (int64_t i = begin + threadIdx.x; i < end; i += blockDim.x) acc[0] += x[i];
    unsigned int *counter = reinterpret_cast<unsigned int *>(scratch + kNaBlocks);
    if (grid_reduce<1>(acc, 1, scratch, counter, sm) && threadIdx.x == 0) out[0] = sm.final_[0];
}

std::mutex g_mu;
std::vector<double *> g_dev_ptr;  // device address of g_sum_scratch, per device

// The symbol's device address, looked up once per device with that device current.
cufsp_status scratch_address(double **out) {
    int dev = 0;
    CUFSP_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_mu);
    if ((int)g_dev_ptr.size() <= dev) g_dev_ptr.resize(dev + 1, nullptr);
    if (!g_dev_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_sum_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cufsp_vec_sum_noalloc: cudaGetSymbolAddress");
        g_dev_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_dev_ptr[dev];
    return CUFSP_SUCCESS;
}

}  // namespace
}  // namespace cufsp

using namespace cufsp;

extern "C" cufsp_status cufsp_vec_sum_noalloc(int64_t n, const double *x, double *d_out, cufsp_stream_t stream) {
    if (!d_out || n < 0 || (n > 0 && !x))  // an empty input may come with a null pointer
        return set_error(CUFSP_ERR_INVALID_ARG, "cufsp_vec_sum_noalloc: bad argument");
    if (n > CUFSP_NOALLOC_MAX_N)
        return set_error(CUFSP_ERR_INVALID_ARG,
                         "cufsp_vec_sum_noalloc: n exceeds CUFSP_NOALLOC_MAX_N (4194304), the size its fixed "
                         "scratch array covers; use cufsp_vec_sum");
    double *scratch = nullptr;
    cufsp_status s = scratch_address(&scratch);
    if (s != CUFSP_SUCCESS) return s;
    cudaStream_t st = (cudaStream_t)stream;
    if (n == 0) {
        CUFSP_CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(double), st));
        return CUFSP_SUCCESS;
    }
    // The array keeps the previous call's contents; only the completion counter must start at 0
    // (the partials are overwritten before they are read).
    CUFSP_CUDA_TRY(cudaMemsetAsync(scratch + kNaBlocks, 0, sizeof(unsigned int), st));
    const int blocks = (int)((n + kNaPerBlock - 1) / kNaPerBlock);
    k_sum_noalloc<<<blocks, kRedThreads, 0, st>>>(n, x, scratch, d_out);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}
