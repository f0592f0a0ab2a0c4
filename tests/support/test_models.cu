// test_models.cu -- device propensity functions for the tests (TEST SUPPORT).
//
// Compiled with -rdc and device-linked together with the cufsp library sources into
// tests/support/libcufsp_testmodels.so, so that the addresses returned below are callable from the
// library's fill kernel (the reference obtains its PropFun the same way:
// cudaMemcpyFromSymbol(&host_prop_ptr, prop_pointer, ...), tests/test_fsp_mat.cu:121-124).
#include <cuda_runtime.h>

#include "cufsp.h"

namespace {
__device__ const double kAyx = 2.6e-3, kAxy = 6.1e-3, kNyx = 3e0, kNxy = 2.1e0;
}

// Toggle switch (tests/test_fsp_mat.cu:19-50).
__device__ double tm_toggle(int *x, int reaction) {
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

// Non-factorisable variant: reactions 1 and 4 couple both species.
__device__ double tm_nonfact(int *x, int reaction) {
    switch (reaction) {
        case 1: return 1.0 / (1.0 + kAyx * pow(1.0 * x[1], kNyx) + 0.05 * x[0]);
        case 4: return (1.0 * x[0]) * (1.0 * x[1]) / (10.0 + x[0] + x[1]) + 1.0;
        default: return tm_toggle(x, reaction);
    }
}

__device__ cufsp_prop_fn tm_toggle_ptr = tm_toggle;
__device__ cufsp_prop_fn tm_nonfact_ptr = tm_nonfact;

extern "C" void *tm_toggle_propfn(void) {
    cufsp_prop_fn p = nullptr;
    if (cudaMemcpyFromSymbol(&p, tm_toggle_ptr, sizeof(p)) != cudaSuccess) return nullptr;
    return (void *)p;
}

extern "C" void *tm_nonfact_propfn(void) {
    cufsp_prop_fn p = nullptr;
    if (cudaMemcpyFromSymbol(&p, tm_nonfact_ptr, sizeof(p)) != cudaSuccess) return nullptr;
    return (void *)p;
}
