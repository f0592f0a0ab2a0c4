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
static int cme_layer();
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

    failures += cme_layer();
    std::printf("%s (%d failures)\n", failures ? "FAILED" : "ok", failures);
    return failures ? 1 : 0;
}

// ---- the legacy cme:: layer (src/Model.h, src/FSPSolver.h, src/Likelihood.h) ------------------------
// A gene-expression network: 3 binary genes, nuclear and cytoplasmic mRNA (12 reactions), box
// (1,1,1,31,31).  The parameters are the 12 rates (t_fun unset).  The program prints the
// log-likelihood and its gradient for the pytest wrapper, which recomputes both with the oracle.
namespace {
double gene_factor(int x, int species, int reaction) {
    if (reaction < 3 && species == reaction) return 1.0 - x;
    if (reaction >= 3 && reaction < 6 && species == reaction - 3) return 1.0 * x;
    if (reaction >= 6 && reaction < 9 && species == reaction - 6) return 1.0 * x;
    if ((reaction == 9 || reaction == 10) && species == 3) return 1.0 * x;
    if (reaction == 11 && species == 4) return 1.0 * x;
    return 1.0;
}
// the same propensities as a host function of a batch of states (the reference's Model::propensity)
void gene_propensity(const int *states, int n_states, int n_species, double *props) {
    for (int k = 0; k < n_states; ++k)
        for (int r = 0; r < 12; ++r) {
            double v = 1.0;
            for (int s = 0; s < n_species; ++s) v *= gene_factor(states[k * n_species + s], s, r);
            props[r * n_states + k] = v;
        }
}
cme::Model gene_model(bool factorised) {
    cme::Model m;
    m.FSPSize = {1, 1, 1, 31, 31};
    m.stoich_mat.assign(5, std::vector<int>(12, 0));
    for (int i = 0; i < 3; ++i) {
        m.stoich_mat[i][i] = 1;
        m.stoich_mat[i][3 + i] = -1;
        m.stoich_mat[3][6 + i] = 1;
    }
    m.stoich_mat[3][9] = -1;
    m.stoich_mat[4][9] = 1;
    m.stoich_mat[3][10] = -1;
    m.stoich_mat[4][11] = -1;
    m.states_init = {{0, 0, 0, 0, 0}};
    m.probs_init = {1.0};
    m.parameters = {0.05, 0.04, 0.03, 2.0, 2.0, 3.0, 0.5, 1.5, 2.0, 0.5, 0.1, 0.05};
    if (factorised) m.prop_factor = &gene_factor;
    else m.propensity = &gene_propensity;
    return m;
}
}  // namespace

static int cme_layer() {
    int fails = 0;
    const std::vector<double> times = {1.0, 3.0, 8.0};
    cme::Model mf = gene_model(true), mh = gene_model(false);
    // FSPSolver through the output times, the factorised and the host-propensity generators
    std::vector<double> pf, ph;
    cme::FSPSolver sf(pf, mf, times, 1e-6), sh(ph, mh, times, 1e-6);
    if (pf.size() != 8192 || pf[0] != 1.0) {
        std::printf("FAIL: FSPSolver initial vector\n");
        ++fails;
    }
    for (size_t it = 0; it < times.size(); ++it) {
        sf.next_time();
        sh.next_time();
        double d = 0.0, mass = 0.0;
        for (size_t i = 0; i < pf.size(); ++i) {
            d += std::fabs(pf[i] - ph[i]);
            mass += pf[i];
        }
        if (!(d <= 1e-8) || std::fabs(sf.current_time() - times[it]) > 0 || !(mass <= 1.0 + 1e-12)) {
            std::printf("FAIL: FSPSolver at t=%g: |p_kron - p_hyb|_1 = %g, mass %.17g\n", times[it], d, mass);
            ++fails;
        }
        if (std::fabs(sf.fsp_error() - (1.0 - mass)) > 1e-12) {
            std::printf("FAIL: fsp_error %g vs 1 - mass %g\n", sf.fsp_error(), 1.0 - mass);
            ++fails;
        }
    }
    const std::vector<double> p_end(pf);
    // reset_time re-reads P: the caller returns it to the initial condition (Likelihood.cpp:24-30)
    std::fill(pf.begin(), pf.end(), 0.0);
    pf[0] = 1.0;
    sf.reset_time();
    sf.solve();
    double dr = 0.0;
    for (size_t i = 0; i < pf.size(); ++i) dr += std::fabs(pf[i] - p_end[i]);
    // solve() steps straight to the last time, so its Krylov steps differ from next_time()'s: the two
    // agree within the Krylov tolerance
    if (!(dr <= 1e-8)) {
        std::printf("FAIL: solve after reset_time differs by %g\n", dr);
        ++fails;
    }
    // data, likelihood and gradient
    cme::SingleCellData data = cme::generate_data(mf, times, {0, 0, 0, 0, 0}, 500, 777ULL);
    if (data.snapshots.size() != times.size() || data.snapshots[0].size() != 500 * 5) {
        std::printf("FAIL: generate_data shape\n");
        ++fails;
    }
    cme::Likelihood L(data, mf);
    L.set_krylov(30, 1e-10);
    const double ll = L.evaluate(mf.parameters);
    double ll_g = 0.0;
    const std::vector<double> g = L.gradient(mf.parameters, &ll_g);
    if (!(std::fabs(ll - ll_g) <= 1e-8 * std::fabs(ll))) {
        std::printf("FAIL: evaluate %.17g vs gradient's log L %.17g\n", ll, ll_g);
        ++fails;
    }
    cme::Likelihood Lh(data, mh);  // the host-propensity model evaluates too (no gradient)
    Lh.set_krylov(30, 1e-10);
    const double llh = Lh.evaluate(mh.parameters);
    if (!(std::fabs(ll - llh) <= 1e-8 * std::fabs(ll))) {
        std::printf("FAIL: log L kron %.17g vs hyb %.17g\n", ll, llh);
        ++fails;
    }
    bool threw = false;
    try {
        Lh.gradient(mh.parameters);
    } catch (const cuFSP::error &e) {
        threw = e.status == CUFSP_ERR_UNSUPPORTED;
    }
    if (!threw) {
        std::printf("FAIL: gradient of a host-propensity model must be refused\n");
        ++fails;
    }
    std::printf("CME logL %.17g\nCME grad", ll);
    for (double v : g) std::printf(" %.17g", v);
    std::printf("\n");
    return fails;
}
