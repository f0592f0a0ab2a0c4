// cufsp.hpp -- C++ drop-in classes with the reference's names and signatures, over the C ABI.
//
//   cuFSP::FSPMat      <- src/FSPMat.h:21-56
//   cuFSP::KryExpvFSP  <- src/KryExpvFSP.h:20-108
//   cuFSP::PropFun, PropFactorFun, TcoefFun, MatrixFormat, CSRMatInt, rect_fsp_num_states,
//   indx2state, state2indx  <- src/cme_util.h:25-62, src/fspmat_kron_kernels.h:13, src/FSPMat.h:16-19
//   cme::Model          <- src/Model.h:14-26
//   cme::FSPSolver      <- src/FSPSolver.h:16-111, src/FSPSolver.cpp:9-22
//   cme::SingleCellData, cme::Likelihood, cme::generate_data <- src/Likelihood.h:15-57, src/Likelihood.cpp:8-84
// The cme:: classes keep the reference's names, constructor arguments and call sequence with
// std::vector in place of the Armadillo types (Armadillo is not a dependency of this library).
//
// Errors throw cuFSP::error (carrying the cufsp_status) instead of exit() (src/cme_util.h:9-22).
// A PropFun (a __device__ function address) is callable by the library only when the program is
// device-linked with the library's relocatable archive (libcufsp_static.a, nvcc -rdc=true).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <stdexcept>
#include <utility>
#include <string>
#include <vector>

#include "cufsp.h"

namespace cuFSP {

class error : public std::runtime_error {
   public:
    cufsp_status status;
    error(cufsp_status s, const char *where)
        : std::runtime_error(std::string(where) + ": " + cufsp_status_string(s) + " (" + cufsp_last_error() + ")"),
          status(s) {}
};

inline void check(cufsp_status s, const char *where) {
    if (s != CUFSP_SUCCESS) throw error(s, where);
}

typedef double (*PropFun)(int *x, int reaction);
typedef double (*PropFactorFun)(int state, int species, int reaction);
typedef std::function<void(double, double *)> TcoefFun;
typedef std::function<void(double *x, double *y)> MVFun;

enum MatrixFormat { CUDA_CSR = CUFSP_FORMAT_CSR, HYB = CUFSP_FORMAT_HYB, KRONECKER = CUFSP_FORMAT_KRONECKER };

struct CSRMatInt {
    int *vals = nullptr;
    int *col_idxs = nullptr;
    int *row_ptrs = nullptr;
    int n_rows = 0, n_cols = 0, nnz = 0;
};

inline int rect_fsp_num_states(int n_species, int *fsp_bounds) {
    int64_t n = 0;
    check(cufsp_num_states(n_species, fsp_bounds, &n), "rect_fsp_num_states");
    return (int)n;
}

inline void indx2state(int indx, int *state, int dim, int *fsp_bounds) {
    check(cufsp_indx2state(indx, state, dim, fsp_bounds), "indx2state");
}

inline int state2indx(int *state, int dim, int *fsp_bounds) {
    int64_t i = 0;
    check(cufsp_state2indx(state, dim, fsp_bounds, &i), "state2indx");
    return (int)i;
}

class FSPMat {
    cufsp_mat *h_ = nullptr;
    TcoefFun tfun_;
    int nr_ = 0, ns_ = 0;
    int64_t n_ = 0;

    static void tcoef_trampoline(double t, double *out, void *user) { (*static_cast<TcoefFun *>(user))(t, out); }

    void create(int n_reactions, int n_species, int *fsp_dim, const CSRMatInt &stoich, TcoefFun t_func,
                PropFun prop, PropFactorFun pff, MatrixFormat format) {
        tfun_ = std::move(t_func);
        nr_ = n_reactions;
        ns_ = n_species;
        cufsp_model_desc d = {};
        d.n_species = n_species;
        d.n_reactions = n_reactions;
        d.fsp_bounds = fsp_dim;
        d.stoich_vals = stoich.vals;
        d.stoich_colidxs = stoich.col_idxs;
        d.stoich_rowptrs = stoich.row_ptrs;
        d.prop_device = prop;
        d.prop_factor = pff;
        if (tfun_) {
            d.tcoef = &FSPMat::tcoef_trampoline;
            d.tcoef_user = &tfun_;
        }
        check(cufsp_mat_create(&d, (cufsp_format)format, &h_), "FSPMat::FSPMat");
        check(cufsp_mat_num_states(h_, &n_), "FSPMat::FSPMat");
    }

   public:
    // src/FSPMat.cu:10-45 (device propensity; CSR or HYB)
    FSPMat(int n_reactions, int n_species, int *fsp_dim, CSRMatInt stoich, TcoefFun t_func, PropFun prop_func,
           MatrixFormat format = CUDA_CSR) {
        create(n_reactions, n_species, fsp_dim, stoich, std::move(t_func), prop_func, nullptr, format);
    }
    // src/FSPMat.cu:49-76 (host factorised propensity; KRONECKER)
    FSPMat(int n_reactions, int n_species, int *fsp_dim, CSRMatInt stoich, TcoefFun t_func, PropFactorFun pffunc,
           MatrixFormat format) {
        create(n_reactions, n_species, fsp_dim, stoich, std::move(t_func), nullptr, pffunc, format);
    }
    FSPMat(const FSPMat &) = delete;
    FSPMat &operator=(const FSPMat &) = delete;
    ~FSPMat() { cufsp_mat_destroy(h_); }

    // y += A(t) x on the legacy default stream (the reference synchronised the device here).
    void action(double t, double *x, double *y) { check(cufsp_mat_action(h_, t, x, y, nullptr), "FSPMat::action"); }

    int get_n_rows() { return (int)n_; }
    int get_n_species() { return ns_; }
    int get_n_reactions() { return nr_; }
    cufsp_mat *handle() { return h_; }
};

class KryExpvFSP {
    cufsp_expv *h_ = nullptr;
    MVFun *mv_ = nullptr;
    FSPMat *A_ = nullptr;
    double t_mat_ = 0.0;
    double *v_ = nullptr;
    int64_t n_ = 0;
    double t_final_, tol_, anorm_;
    int built_m_ = -1, built_iop_ = -1, built_q_ = -1;

    static double *raw_ptr(double *p) { return p; }
    template <class Ptr>
    static double *raw_ptr(Ptr p) {  // a fancy device pointer (thrust::device_ptr and the like)
        return p.get();
    }

    static int mv_trampoline(const double *x, double *y, void *user, cufsp_stream_t) {
        try {
            (*static_cast<MVFun *>(user))(const_cast<double *>(x), y);
            return 0;
        } catch (...) {
            return 1;
        }
    }

    // The handle is built from the public members (m, IOP, q_iop, max_nstep, max_reject -- public
    // fields in the reference too) at the first solve()/step(); the limits may change later, the
    // Krylov shape may not (that throws CUFSP_ERR_UNSUPPORTED).
    void ensure() {
        if (h_) {
            if (built_m_ != m || built_iop_ != (int)IOP || built_q_ != q_iop)
                throw error(CUFSP_ERR_UNSUPPORTED, "KryExpvFSP: m / IOP / q_iop changed after the first step");
            check(cufsp_expv_set_limits(h_, max_nstep, max_reject), "KryExpvFSP");
            return;
        }
        check(cufsp_expv_create(n_, m, tol_, IOP ? 1 : 0, q_iop, anorm_, &h_), "KryExpvFSP");
        if (A_) check(cufsp_expv_bind_mat(h_, A_->handle(), t_mat_), "KryExpvFSP");
        else check(cufsp_expv_bind_matvec(h_, &KryExpvFSP::mv_trampoline, mv_), "KryExpvFSP");
        check(cufsp_expv_set_final_time(h_, t_final_), "KryExpvFSP");
        check(cufsp_expv_set_limits(h_, max_nstep, max_reject), "KryExpvFSP");
        built_m_ = m;
        built_iop_ = IOP;
        built_q_ = q_iop;
    }

   public:
    bool IOP = false;
    int q_iop = 2;
    int m = 30;
    int max_nstep = 10000;
    int max_reject = 1000;

    // src/KryExpvFSP.h:75-76 with the vector as a device pointer and its length
    KryExpvFSP(double t_final, MVFun &matvec, double *v, int64_t n, int m_, double tol = 1.0e-8, bool iop = false,
               int q = 2, double anorm = 1.0)
        : mv_(&matvec), v_(v), n_(n), t_final_(t_final), tol_(tol), anorm_(anorm), IOP(iop), q_iop(q), m(m_) {}
    // generator fast path: the action of A(t_mat) is applied without a callback
    KryExpvFSP(double t_final, FSPMat &A, double t_mat, double *v, int m_, double tol = 1.0e-8, bool iop = false,
               int q = 2, double anorm = 1.0)
        : A_(&A), t_mat_(t_mat), v_(v), n_(A.get_n_rows()), t_final_(t_final), tol_(tol), anorm_(anorm), IOP(iop),
          q_iop(q), m(m_) {}
    // the reference's signature (src/KryExpvFSP.h:75-76): v is a device vector with data() and size(),
    // e.g. thrust::device_vector<double> (whose data() is a device_ptr: raw_ptr takes its address)
    template <class DVec, class = decltype(std::declval<DVec &>().data()), class = decltype(std::declval<DVec &>().size())>
    KryExpvFSP(double t_final, MVFun &matvec, DVec &v, int m_, double tol = 1.0e-8, bool iop = false, int q = 2,
               double anorm = 1.0)
        : KryExpvFSP(t_final, matvec, raw_ptr(v.data()), (int64_t)v.size(), m_, tol, iop, q, anorm) {}
    KryExpvFSP(const KryExpvFSP &) = delete;
    KryExpvFSP &operator=(const KryExpvFSP &) = delete;
    ~KryExpvFSP() { cufsp_expv_destroy(h_); }

    void solve() {
        ensure();
        check(cufsp_expv_solve(h_, v_, nullptr, nullptr), "KryExpvFSP::solve");
    }
    void step() {
        ensure();
        check(cufsp_expv_step(h_, v_, nullptr), "KryExpvFSP::step");
    }
    void reset_time() {
        ensure();
        check(cufsp_expv_reset_time(h_), "KryExpvFSP::reset_time");
    }
    bool final_time_reached() {
        ensure();
        int r = 0;
        check(cufsp_expv_final_time_reached(h_, &r), "KryExpvFSP::final_time_reached");
        return r != 0;
    }
    cufsp_expv_stats stats() {
        ensure();
        cufsp_expv_stats st;
        check(cufsp_expv_get_stats(h_, &st), "KryExpvFSP::stats");
        return st;
    }
};

}  // namespace cuFSP

namespace cme {

using cuFSP::check;

// src/Model.h:14-26.  The reference's Armadillo members become std::vector:
//   states_init   initial states, one std::vector<int> of species counts each (Mat<int>, column-wise)
//   probs_init    their probabilities
//   FSPSize       the box bounds b_s (Row<size_t>)
//   stoich_mat    stoich_mat[s][r]: net change of species s by reaction r (Mat<int>, species x reactions)
//   propensity    host propensities of a batch of states: states[k * n_species + s] for k < n_states,
//                 props[r * n_states + k] = a_r(state k)  (the reference's Mat<double>(*)(Mat<int>));
//                 the generator is built from them in the CSR/HYB format
//   prop_factor   alternatively the factorised form a_r(x) = prod_s f(x_s, s, r): KRONECKER format,
//                 matrix-free, and the adjoint gradient
//   t_fun         c(t, parameters), one coefficient per reaction (Row<double>(*)(double, Row<double>))
//   parameters
struct Model {
    typedef void (*PropFun)(const int *states, int n_states, int n_species, double *props);
    typedef std::vector<double> (*InputFun)(double t, const std::vector<double> &parameters);

    std::vector<std::vector<int>> states_init;
    std::vector<double> probs_init;
    std::vector<int> FSPSize;
    std::vector<std::vector<int>> stoich_mat;
    PropFun propensity = nullptr;
    cuFSP::PropFactorFun prop_factor = nullptr;
    InputFun t_fun = nullptr;
    std::vector<double> parameters;

    int n_species() const { return (int)FSPSize.size(); }
    int n_reactions() const { return stoich_mat.empty() ? 0 : (int)stoich_mat[0].size(); }
    int64_t n_states() const {
        int64_t n = 1;
        for (int b : FSPSize) n *= (int64_t)b + 1;
        return n;
    }
    // index of a state in the box (species 0 fastest), -1 outside (sub2ind_fsp of the reference)
    int64_t index(const int *x) const {
        int64_t i = 0, stride = 1;
        for (size_t s = 0; s < FSPSize.size(); ++s) {
            if (x[s] < 0 || x[s] > FSPSize[s]) return -1;
            i += (int64_t)x[s] * stride;
            stride *= (int64_t)FSPSize[s] + 1;
        }
        return i;
    }
    std::vector<double> coefficients(double t, const std::vector<double> &params) const {
        if (!t_fun) return params;
        std::vector<double> c = t_fun(t, params);
        if ((int)c.size() != n_reactions()) throw cuFSP::error(CUFSP_ERR_INVALID_ARG, "cme::Model::t_fun size");
        return c;
    }
};

namespace detail {
// The generator of a Model: KRONECKER from prop_factor, else HYB from the host propensities.
class Generator {
    cufsp_mat *h_ = nullptr;

   public:
    explicit Generator(const Model &model) {
        const int ns = model.n_species(), nr = model.n_reactions();
        if (ns < 1 || nr < 1 || (int)model.stoich_mat.size() != ns)
            throw cuFSP::error(CUFSP_ERR_INVALID_ARG, "cme::Model: FSPSize and stoich_mat disagree");
        std::vector<int> vals, cols, rows{0};
        for (int r = 0; r < nr; ++r) {
            for (int s = 0; s < ns; ++s)
                if (model.stoich_mat[s][r] != 0) {
                    vals.push_back(model.stoich_mat[s][r]);
                    cols.push_back(s);
                }
            rows.push_back((int)vals.size());
        }
        std::vector<int> bounds(model.FSPSize);
        cufsp_model_desc d = {};
        d.n_species = ns;
        d.n_reactions = nr;
        d.fsp_bounds = bounds.data();
        d.stoich_vals = vals.data();
        d.stoich_colidxs = cols.data();
        d.stoich_rowptrs = rows.data();
        if (model.prop_factor) {
            d.prop_factor = model.prop_factor;
            check(cufsp_mat_create(&d, CUFSP_FORMAT_KRONECKER, &h_), "cme::Model generator");
        } else if (model.propensity) {
            const int64_t n = model.n_states();
            std::vector<int> states((size_t)n * ns);
            for (int64_t k = 0; k < n; ++k) check(cufsp_indx2state(k, &states[(size_t)k * ns], ns, bounds.data()), "cme");
            std::vector<double> props((size_t)n * nr);
            model.propensity(states.data(), (int)n, ns, props.data());
            check(cufsp_mat_create_table(&d, CUFSP_FORMAT_HYB, props.data(), &h_), "cme::Model generator");
        } else {
            throw cuFSP::error(CUFSP_ERR_INVALID_ARG, "cme::Model: neither propensity nor prop_factor is set");
        }
    }
    Generator(const Generator &) = delete;
    Generator &operator=(const Generator &) = delete;
    ~Generator() { cufsp_mat_destroy(h_); }
    cufsp_mat *get() const { return h_; }
};

// A device copy of a host vector.
class DeviceVector {
    double *d_ = nullptr;
    size_t n_ = 0;

   public:
    explicit DeviceVector(size_t n) : n_(n) {
        if (cudaMalloc(&d_, sizeof(double) * std::max<size_t>(1, n)) != cudaSuccess)
            throw cuFSP::error(CUFSP_ERR_ALLOC, "cme: device vector");
    }
    DeviceVector(const DeviceVector &) = delete;
    DeviceVector &operator=(const DeviceVector &) = delete;
    ~DeviceVector() { cudaFree(d_); }
    double *get() const { return d_; }
    void upload(const double *h) {
        if (cudaMemcpy(d_, h, sizeof(double) * n_, cudaMemcpyHostToDevice) != cudaSuccess)
            throw cuFSP::error(CUFSP_ERR_CUDA, "cme: upload");
    }
    void download(double *h) const {
        if (cudaMemcpy(h, d_, sizeof(double) * n_, cudaMemcpyDeviceToHost) != cudaSuccess)
            throw cuFSP::error(CUFSP_ERR_CUDA, "cme: download");
    }
};

inline void initial_distribution(const Model &model, std::vector<double> &p) {
    const int64_t n = model.n_states();
    if ((int64_t)p.size() >= n) return;  // the caller's vector is kept (src/FSPSolver.h:46-57)
    p.assign((size_t)n, 0.0);
    for (size_t i = 0; i < model.states_init.size() && i < model.probs_init.size(); ++i) {
        const int64_t k = model.index(model.states_init[i].data());
        if (k < 0) throw cuFSP::error(CUFSP_ERR_INVALID_ARG, "cme: initial state outside the FSP box");
        p[(size_t)k] = model.probs_init[i];
    }
}
}  // namespace detail

// src/FSPSolver.h:16-111.  P is the caller's host vector (resized and set from the model's initial
// states when it is smaller than the box, as the reference does); next_time() advances it to the next
// output time with the Krylov exponential of A(t = 0) (the reference binds A(0); IOP with q = 2, m = 30),
// solve() goes to the last time, reset_time() returns to t = 0 and reads P again at the next advance.
// fsp_error() is the probability that has left the box (the reference stores fsp_tol but never uses it;
// fsp_tol_exceeded() compares with it).  mg_tol is accepted for the signature and unused, as there.
class FSPSolver {
    const Model &model_;
    std::vector<double> &P;
    std::vector<double> times_;
    double fsp_tol_;
    detail::Generator A_;
    detail::DeviceVector d_p_;
    cufsp_solver *h_ = nullptr;
    cufsp_solver_status st_ = {};
    bool upload_ = true;

   public:
    FSPSolver(std::vector<double> &_p, const Model &_model, const std::vector<double> &_times, double _fsp_tol,
              double _mg_tol = 1.0e-8, double _kry_tol = 1.0e-8)
        : model_(_model), P(_p), times_(_times), fsp_tol_(_fsp_tol), A_(_model),
          d_p_((size_t)_model.n_states()) {
        (void)_mg_tol;
        detail::initial_distribution(model_, P);
        const std::vector<double> c = model_.coefficients(0.0, model_.parameters);
        check(cufsp_solver_create(A_.get(), times_.data(), (int)times_.size(), fsp_tol_, c.data(), _kry_tol, 30, 1, 2,
                                  &h_),
              "cme::FSPSolver");
    }
    FSPSolver(std::vector<double> &_p, const Model &_model, double _t_final, double _fsp_tol, double _mg_tol = 1.0e-8,
              double _kry_tol = 1.0e-8)
        : FSPSolver(_p, _model, std::vector<double>{_t_final}, _fsp_tol, _mg_tol, _kry_tol) {}
    FSPSolver(const FSPSolver &) = delete;
    FSPSolver &operator=(const FSPSolver &) = delete;
    ~FSPSolver() { cufsp_solver_destroy(h_); }

    // src/FSPSolver.cpp:11-17
    void next_time() {
        prepare();
        check(cufsp_solver_next_time(h_, d_p_.get(), nullptr, &st_), "cme::FSPSolver::next_time");
        d_p_.download(P.data());
    }
    // src/FSPSolver.cpp:19-22
    void solve() {
        prepare();
        check(cufsp_solver_solve(h_, d_p_.get(), nullptr, &st_), "cme::FSPSolver::solve");
        d_p_.download(P.data());
    }
    // src/FSPSolver.h:99-105
    void reset_time() {
        check(cufsp_solver_reset_time(h_), "cme::FSPSolver::reset_time");
        upload_ = true;
    }
    // new coefficients c = t_fun(0, parameters) for the next advances
    void set_parameters(const std::vector<double> &parameters) {
        const std::vector<double> c = model_.coefficients(0.0, parameters);
        check(cufsp_solver_set_coefs(h_, c.data()), "cme::FSPSolver::set_parameters");
    }
    double current_time() const { return st_.t; }
    double fsp_error() const { return st_.fsp_error; }
    bool fsp_tol_exceeded() const { return st_.fsp_error > fsp_tol_; }
    cufsp_mat *generator() const { return A_.get(); }

   private:
    void prepare() {
        if ((int64_t)P.size() != model_.n_states())
            throw cuFSP::error(CUFSP_ERR_INVALID_ARG, "cme::FSPSolver: P does not match the FSP box");
        if (upload_) {
            d_p_.upload(P.data());
            upload_ = false;
        }
    }
};

// src/Likelihood.h:15-19: snapshots[it][cell * n_species + s] is species s of cell `cell` at times[it]
// (the reference's field<Mat<int>>, one species x cells matrix per time).
struct SingleCellData {
    std::vector<double> times;
    std::vector<std::vector<int>> snapshots;
};

// src/Likelihood.h:23-53, src/Likelihood.cpp:8-33.  evaluate(parameters) returns
//   sum_t sum_cells log max(1e-44, p_t(x_cell)),  p_t = exp(t A(c)) p0,  c = t_fun(0, parameters),
// on the full joint state as the reference does; a cell outside the FSP box contributes log(1e-44).
// The whole pass runs on the device in one call (cufsp_likelihood_eval).  gradient(parameters)
// returns d log L / d parameters by the adjoint method (cufsp_likelihood_grad; no counterpart in the
// reference): it needs the factorised propensity (prop_factor), and the chain rule through t_fun
// takes its Jacobian at t = 0 by central differences (relative step 1e-6).
class Likelihood {
   protected:
    SingleCellData &data;
    Model &model;
    detail::Generator A_;
    detail::DeviceVector d_p0_, d_counts_;
    double outside_ = 0.0;  // cells outside the box
    int m_ = 30;
    double kry_tol_ = 1.0e-8;

   public:
    Likelihood(SingleCellData &_data, Model &_model)
        : data(_data), model(_model), A_(_model), d_p0_((size_t)_model.n_states()),
          d_counts_((size_t)_model.n_states() * std::max<size_t>(1, _data.times.size())) {
        const int ns = model.n_species();
        const int64_t n = model.n_states();
        if (data.snapshots.size() != data.times.size())
            throw cuFSP::error(CUFSP_ERR_INVALID_ARG, "cme::Likelihood: one snapshot per time");
        std::vector<double> counts((size_t)n * data.times.size(), 0.0);
        for (size_t it = 0; it < data.times.size(); ++it) {  // data2fsp (src/Likelihood.h:35-41)
            const std::vector<int> &snap = data.snapshots[it];
            for (size_t c = 0; c + ns <= snap.size(); c += ns) {
                const int64_t k = model.index(&snap[c]);
                if (k < 0) outside_ += 1.0;
                else counts[it * (size_t)n + (size_t)k] += 1.0;
            }
        }
        d_counts_.upload(counts.data());
        std::vector<double> p0;
        detail::initial_distribution(model, p0);
        d_p0_.upload(p0.data());
    }

    // Krylov settings of the forward solve (and of the gradient's forward and backward solves)
    void set_krylov(int m, double tol) {
        m_ = m;
        kry_tol_ = tol;
    }

    double evaluate(const std::vector<double> &parameters) {
        model.parameters = parameters;
        const std::vector<double> c = model.coefficients(0.0, parameters);
        double ll = 0.0;
        check(cufsp_likelihood_eval(A_.get(), c.data(), (int)data.times.size(), data.times.data(), d_p0_.get(), 1,
                                    d_counts_.get(), m_, kry_tol_, &ll, nullptr, nullptr),
              "cme::Likelihood::evaluate");
        return ll + outside_ * std::log(1.0e-44);
    }

    std::vector<double> gradient(const std::vector<double> &parameters, double *logL = nullptr) {
        if (!model.prop_factor)
            throw cuFSP::error(CUFSP_ERR_UNSUPPORTED, "cme::Likelihood::gradient needs the factorised propensity");
        const int nr = model.n_reactions();
        const std::vector<double> c = model.coefficients(0.0, parameters);
        std::vector<double> g(nr);
        double ll = 0.0;
        check(cufsp_likelihood_grad(A_.get(), c.data(), (int)data.times.size(), data.times.data(), d_p0_.get(), 1,
                                    d_counts_.get(), m_, kry_tol_, &ll, g.data(), nullptr),
              "cme::Likelihood::gradient");
        if (logL) *logL = ll + outside_ * std::log(1.0e-44);
        // d log L / d c_r = g_r / c_r, then through t_fun
        const size_t np = parameters.size();
        std::vector<double> out(np, 0.0);
        for (size_t k = 0; k < np; ++k) {
            std::vector<double> dc(nr, 0.0);
            if (!model.t_fun) {
                if ((int)np != nr) throw cuFSP::error(CUFSP_ERR_INVALID_ARG, "cme::Likelihood: parameters are the rates");
                dc[k] = 1.0;
            } else {
                const double h = 1e-6 * std::max(1.0, std::fabs(parameters[k]));
                std::vector<double> pp(parameters), pm(parameters);
                pp[k] += h;
                pm[k] -= h;
                const std::vector<double> cp = model.coefficients(0.0, pp), cm = model.coefficients(0.0, pm);
                for (int r = 0; r < nr; ++r) dc[r] = (cp[r] - cm[r]) / (2.0 * h);
            }
            for (int r = 0; r < nr; ++r) {
                if (dc[r] == 0.0) continue;
                if (c[r] == 0.0)
                    throw cuFSP::error(CUFSP_ERR_UNSUPPORTED, "cme::Likelihood::gradient: a rate is zero");
                out[k] += g[r] / c[r] * dc[r];
            }
        }
        return out;
    }
};

// src/Likelihood.cpp:35-84: num_samples single-cell snapshots per time, an independent trajectory
// from x0 for each (time, cell), with seeded counter-based streams (the reference draws unseeded).
// Needs the factorised propensity (the SSA evaluates a_r from the factor tables).
inline SingleCellData generate_data(Model &model, const std::vector<double> &times, const std::vector<int> &x0,
                                    size_t num_samples, unsigned long long seed = 20261203ULL) {
    if (!model.prop_factor)
        throw cuFSP::error(CUFSP_ERR_UNSUPPORTED, "cme::generate_data needs the factorised propensity");
    const int ns = model.n_species(), nr = model.n_reactions();
    std::vector<int> vals, cols, rows{0};
    for (int r = 0; r < nr; ++r) {
        for (int s = 0; s < ns; ++s)
            if (model.stoich_mat[s][r] != 0) {
                vals.push_back(model.stoich_mat[s][r]);
                cols.push_back(s);
            }
        rows.push_back((int)vals.size());
    }
    std::vector<int> bounds(model.FSPSize);
    cufsp_model_desc d = {};
    d.n_species = ns;
    d.n_reactions = nr;
    d.fsp_bounds = bounds.data();
    d.stoich_vals = vals.data();
    d.stoich_colidxs = cols.data();
    d.stoich_rowptrs = rows.data();
    d.prop_factor = model.prop_factor;
    const std::vector<double> c = model.coefficients(0.0, model.parameters);
    const size_t total = times.size() * num_samples * (size_t)ns;
    int *d_out = nullptr;
    if (cudaMalloc(&d_out, sizeof(int) * std::max<size_t>(1, total)) != cudaSuccess)
        throw cuFSP::error(CUFSP_ERR_ALLOC, "cme::generate_data");
    const cufsp_status s = cufsp_ssa(&d, c.data(), x0.data(), times.data(), (int)times.size(), (int)num_samples, seed,
                                     100000000LL, d_out, nullptr);
    std::vector<int> all(total);
    if (s == CUFSP_SUCCESS) cudaMemcpy(all.data(), d_out, sizeof(int) * total, cudaMemcpyDeviceToHost);
    cudaFree(d_out);
    check(s, "cme::generate_data");
    SingleCellData out;
    out.times = times;
    for (size_t it = 0; it < times.size(); ++it)
        out.snapshots.emplace_back(all.begin() + it * num_samples * ns, all.begin() + (it + 1) * num_samples * ns);
    return out;
}

}  // namespace cme
