// cufsp.hpp -- C++ drop-in classes with the reference's names and signatures, over the C ABI.
//
//   cuFSP::FSPMat      <- src/FSPMat.h:21-56
//   cuFSP::KryExpvFSP  <- src/KryExpvFSP.h:20-108
//   cuFSP::PropFun, PropFactorFun, TcoefFun, MatrixFormat, CSRMatInt, rect_fsp_num_states,
//   indx2state, state2indx  <- src/cme_util.h:25-62, src/fspmat_kron_kernels.h:13, src/FSPMat.h:16-19
//
// Errors throw cuFSP::error (carrying the cufsp_status) instead of exit() (src/cme_util.h:9-22).
// A PropFun (a __device__ function address) is callable by the library only when the program is
// device-linked with the library's relocatable archive (libcufsp_static.a, nvcc -rdc=true).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <stdexcept>
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
#if defined(THRUST_VERSION)
    // the reference's signature: thrust::device_vector<double> &v
    template <class DVec>
    KryExpvFSP(double t_final, MVFun &matvec, DVec &v, int m_, double tol = 1.0e-8, bool iop = false, int q = 2,
               double anorm = 1.0)
        : KryExpvFSP(t_final, matvec, thrust::raw_pointer_cast(v.data()), (int64_t)v.size(), m_, tol, iop, q, anorm) {}
#endif
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
