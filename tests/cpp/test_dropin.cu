// test_dropin.cu -- the reference's own usage pattern, compiled against include/cufsp.hpp.
//
// Follows the flow of the reference tests (tests/test_fsp_mat.cu, tests/test_kry_expv.cu): a
// two-gene toggle switch, a __device__ propensity whose address is fetched with
// cudaMemcpyFromSymbol, a host factorised propensity for the KRONECKER format, thrust device
// vectors, and an MVFun lambda around FSPMat::action.  Built with nvcc -rdc=true and linked with
// libcufsp_static.a so the device propensity is callable by the library.  Exit code 0 = pass.
#include <thrust/device_vector.h>
#include <thrust/fill.h>
#include <thrust/reduce.h>
#include <thrust/transform.h>

#include <cmath>
#include <cstdio>

#include "cufsp.hpp"

namespace {
const double ayx = 2.6e-3, axy = 6.1e-3, nyx = 3e0, nxy = 2.1e0, kx0 = 2.2e-3, kx = 1.7e-2, dx = 3.8e-4,
             ky0 = 6.8e-5, ky = 1.6e-2, dy = 3.8e-4;
}

__device__ double toggle_prop(int *x, int reaction) {
    switch (reaction) {
        case 0: return 1.0;
        case 1: return 1.0 / (1.0 + ayx * pow(1.0 * x[1], nyx));
        case 2: return 1.0 * x[0];
        case 3: return 1.0;
        case 4: return 1.0 / (1.0 + axy * pow(1.0 * x[0], nxy));
        case 5: return 1.0 * x[1];
        default: return 0.0;
    }
}
__device__ cuFSP::PropFun toggle_prop_ptr = toggle_prop;

double toggle_factor(int x, int species, int reaction) {
    if (reaction == 1 && species == 1) return 1.0 / (1.0 + ayx * std::pow(1.0 * x, nyx));
    if (reaction == 2 && species == 0) return 1.0 * x;
    if (reaction == 4 && species == 0) return 1.0 / (1.0 + axy * std::pow(1.0 * x, nxy));
    if (reaction == 5 && species == 1) return 1.0 * x;
    return 1.0;
}

void t_func(double, double *out) {
    out[0] = kx0;
    out[1] = kx;
    out[2] = dx;
    out[3] = ky0;
    out[4] = ky;
    out[5] = dy;
}

static int failures = 0;
#define EXPECT(cond, ...)                      \
    do {                                       \
        if (!(cond)) {                         \
            std::printf("FAIL: " __VA_ARGS__); \
            std::printf("\n");                 \
            ++failures;                        \
        }                                      \
    } while (0)

static double *raw(thrust::device_vector<double> &v) { return thrust::raw_pointer_cast(v.data()); }

static double l2diff(thrust::device_vector<double> &a, thrust::device_vector<double> &b) {
    thrust::device_vector<double> d(a.size());
    thrust::transform(a.begin(), a.end(), b.begin(), d.begin(), [] __device__(double p, double q) { return (p - q) * (p - q); });
    return std::sqrt(thrust::reduce(d.begin(), d.end()));
}

int main() {
    int sv[] = {1, 1, -1, 1, 1, -1}, sc[] = {0, 0, 0, 1, 1, 1}, sr[] = {0, 1, 2, 3, 4, 5, 6};
    cuFSP::CSRMatInt stoich;
    stoich.vals = sv;
    stoich.col_idxs = sc;
    stoich.row_ptrs = sr;
    stoich.n_rows = 6;
    stoich.n_cols = 2;
    stoich.nnz = 6;

    cuFSP::PropFun prop = nullptr;
    cudaMemcpyFromSymbol(&prop, toggle_prop_ptr, sizeof(cuFSP::PropFun));

    // ---- generator formats agree (tests/test_fsp_mat.cu:126-201) ----
    int b31[] = {31, 31};
    const int n = cuFSP::rect_fsp_num_states(2, b31);
    EXPECT(n == 1024, "rect_fsp_num_states = %d", n);
    cuFSP::FSPMat A(6, 2, b31, stoich, &t_func, prop);
    cuFSP::FSPMat A2(6, 2, b31, stoich, &t_func, prop, cuFSP::HYB);
    cuFSP::FSPMat A3(6, 2, b31, stoich, &t_func, &toggle_factor, cuFSP::KRONECKER);
    thrust::device_vector<double> v(n, 0.0), w(n, 0.0), w2(n, 0.0), w3(n, 0.0);
    A.action(1.0, raw(v), raw(w));
    A2.action(1.0, raw(v), raw(w2));
    A3.action(1.0, raw(v), raw(w3));
    cudaDeviceSynchronize();
    EXPECT(std::fabs(thrust::reduce(w.begin(), w.end())) <= 1e-14, "A*0 (CSR)");
    EXPECT(std::fabs(thrust::reduce(w2.begin(), w2.end())) <= 1e-14, "A*0 (HYB)");
    EXPECT(std::fabs(thrust::reduce(w3.begin(), w3.end())) <= 1e-14, "A*0 (KRONECKER)");
    thrust::fill(v.begin(), v.end(), 1.0);
    A.action(1.0, raw(v), raw(w));
    A2.action(1.0, raw(v), raw(w2));
    A3.action(1.0, raw(v), raw(w3));
    cudaDeviceSynchronize();
    const double e12 = l2diff(w, w2), e32 = l2diff(w3, w2);
    EXPECT(e12 <= 1e-14, "||CSR - HYB|| = %g", e12);
    EXPECT(e32 <= 1e-12, "||KRON - HYB|| = %g", e32);
    EXPECT(A.get_n_rows() == n && A.get_n_species() == 2 && A.get_n_reactions() == 6, "getters");

    // ---- Krylov mass conservation (tests/test_kry_expv.cu:80-110) ----
    int b256[] = {1 << 8, 1 << 8};
    cuFSP::FSPMat K(6, 2, b256, stoich, &t_func, prop, cuFSP::HYB);
    const int nk = K.get_n_rows();
    thrust::device_vector<double> p(nk, 0.0);
    p[0] = 1.0;
    cuFSP::MVFun matvec = [&](double *x, double *y) { K.action(1.0, x, y); };
    cuFSP::KryExpvFSP expv(8 * 3600.0, matvec, p, 30, 1.0e-8, true);
    expv.solve();
    cudaDeviceSynchronize();
    const double mass = thrust::reduce(p.begin(), p.end());
    EXPECT(std::fabs(1.0 - mass) <= 1e-10, "mass after expv (MVFun) = %.17g", mass);
    EXPECT(expv.final_time_reached(), "final time reached");

    // same solve through the generator fast path
    thrust::device_vector<double> p2(nk, 0.0);
    p2[0] = 1.0;
    cuFSP::KryExpvFSP expv2(8 * 3600.0, K, 1.0, raw(p2), 30, 1.0e-8, true);
    expv2.solve();
    cudaDeviceSynchronize();
    const double mass2 = thrust::reduce(p2.begin(), p2.end());
    EXPECT(std::fabs(1.0 - mass2) <= 1e-10, "mass after expv (fast path) = %.17g", mass2);
    thrust::device_vector<double> d(nk);
    thrust::transform(p.begin(), p.end(), p2.begin(), d.begin(), [] __device__(double a, double b) { return fabs(a - b); });
    const double diff = thrust::reduce(d.begin(), d.end());
    EXPECT(diff <= 1.2e-8 * 8 * 3600.0, "||p_MVFun - p_fast||_1 = %g", diff);

    // errors are exceptions, not exit()
    bool threw = false;
    try {
        int bad[] = {31, -1};
        cuFSP::FSPMat B(6, 2, bad, stoich, &t_func, &toggle_factor, cuFSP::KRONECKER);
    } catch (const cuFSP::error &e) {
        threw = e.status == CUFSP_ERR_INVALID_ARG;
    }
    EXPECT(threw, "invalid bounds throw cuFSP::error");

    std::printf("%s (%d failures)\n", failures ? "FAILED" : "ok", failures);
    return failures ? 1 : 0;
}
