"""FP64 host oracle for the FSP generator path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py may import this package.
It wraps:
  liboracle.so  -- fsp_oracle.c, a plain-C/OpenMP restatement of the reference's state indexing,
                   per-reaction CSR assembly, SpMV, Krylov expv and the Pade(13) exponential;
  _ref/libref.so -- (optional) the reference's own cme_util/HYB/Kronecker sources compiled by the
                   Makefile in this directory, used to pin the restatement (host functions) and,
                   on a GPU, to compare against the reference kernels.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libref.so"

_I = C.c_int
_I64 = C.c_int64
_P = C.c_void_p
_D = C.c_double


class ExpvStats(C.Structure):
    _fields_ = [("n_steps", C.c_int64), ("n_reject", C.c_int64), ("n_matvec", C.c_int64), ("t_now", C.c_double),
                ("last_err", C.c_double), ("n_breakdown", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BdfStats(C.Structure):
    _fields_ = [("t", C.c_double), ("h", C.c_double), ("last_err", C.c_double), ("order", C.c_int),
                ("pad", C.c_int), ("n_steps", C.c_int64), ("n_reject", C.c_int64), ("n_matvec", C.c_int64),
                ("n_lin_iters", C.c_int64), ("n_lin_fail", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


TCOEF_FN = C.CFUNCTYPE(None, C.c_double, C.POINTER(C.c_double), C.c_void_p)

_lib = None
_ref = None


def build(ref: bool = False) -> None:
    """Compile the oracle (and the reference shim when the reference sources exist)."""
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", str(HERE)] + targets, check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            build()
        L = C.CDLL(str(ORACLE_SO))
        L.orc_num_states.restype = _I64
        L.orc_num_states.argtypes = [_I, _P]
        L.orc_indx2state.argtypes = [_I64, _P, _I, _P]
        L.orc_state2indx.restype = _I64
        L.orc_state2indx.argtypes = [_P, _I, _P]
        L.orc_get_states.argtypes = [_I, _P, _P]
        L.orc_propensity.restype = _D
        L.orc_propensity.argtypes = [_I, _I, _P, _P, _P, _I]
        L.orc_toggle_factor_tables.argtypes = [_P, _P]
        L.orc_assemble_csr.restype = _I
        L.orc_assemble_csr.argtypes = [_I, _I, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P]
        L.orc_spmv.argtypes = [_I64, _I, _P, _P, _P, _P, _P, _D, _P]
        L.orc_abs_spmv.argtypes = [_I64, _I, _P, _P, _P, _P, _P, _P]
        L.orc_norm1.restype = _D
        L.orc_norm1.argtypes = [_I64, _I, _P, _P, _P, _P]
        L.orc_expm.restype = _I
        L.orc_expm.argtypes = [_I, _P, _P]
        L.orc_expv.restype = _I
        L.orc_expv.argtypes = [_I64, _I, _P, _P, _P, _P, _D, _P, _I, _D, _I, _I, _D, _I64, _I64, C.POINTER(ExpvStats)]
        L.orc_num_threads.restype = _I
        L.orc_bdf.restype = _I
        L.orc_bdf.argtypes = [_I64, _I, _P, _P, _P, _P, TCOEF_FN, _P, _D, _P, _P, _I, _P, _D, _D, _I, _D, _D, _D,
                              _I64, C.POINTER(BdfStats)]
        L.orc_bdf_change_matrix.argtypes = [_I, _D, _P]
        _lib = L
    return _lib


def ref() -> C.CDLL | None:
    """The reference's own compiled host/GPU functions, or None when not built."""
    global _ref
    if _ref is None and REF_SO.exists():
        R = C.CDLL(str(REF_SO))
        R.ref_num_states.restype = _I
        R.ref_num_states.argtypes = [_I, _P]
        R.ref_indx2state.argtypes = [_I, _P, _I, _P]
        R.ref_state2indx.restype = _I
        R.ref_state2indx.argtypes = [_P, _I, _P]
        R.ref_sdkron_fill.argtypes = [_I, _P, _I, _P, _P, _P, _P, _P, _P]
        R.ref_gpu_get_states.restype = _I
        R.ref_gpu_get_states.argtypes = [_I, _P, _P]
        R.ref_gpu_hyb_toggle.restype = _I
        R.ref_gpu_hyb_toggle.argtypes = [_P, _P, _P, _P]
        R.ref_gpu_kron.restype = _I
        R.ref_gpu_kron.argtypes = [_I, _I, _P, _P, _P, _P, _P, _P, _P, _P]
        R.ref_gpu_hyb_tables.restype = _I
        R.ref_gpu_hyb_tables.argtypes = [_I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P]
        R.ref_gpu_kron_time.restype = _D
        R.ref_gpu_kron_time.argtypes = [_I, _I, _P, _P, _P, _P, _P, _P, _I]
        _ref = R
    return _ref


def _a(x, dt):
    return np.ascontiguousarray(np.asarray(x, dtype=dt))


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def num_threads() -> int:
    return int(lib().orc_num_threads())


def num_states(bounds) -> int:
    b = _a(bounds, np.int32)
    return int(lib().orc_num_states(len(b), _p(b)))


def get_states(bounds) -> np.ndarray:
    b = _a(bounds, np.int32)
    n = num_states(b)
    out = np.empty((n, len(b)), np.int32)
    lib().orc_get_states(len(b), _p(b), _p(out))
    return out


def indx2state(i: int, bounds) -> np.ndarray:
    b = _a(bounds, np.int32)
    s = np.empty(len(b), np.int32)
    lib().orc_indx2state(int(i), _p(s), len(b), _p(b))
    return s


def state2indx(state, bounds) -> int:
    b = _a(bounds, np.int32)
    s = _a(state, np.int32)
    return int(lib().orc_state2indx(_p(s), len(b), _p(b)))


PROP_TABLES, PROP_TOGGLE, PROP_NONFACT = 0, 1, 2


@dataclass
class CSR:
    """Per-reaction CSR matrices A_r (src/fspmat_csr_kernels.cu:138-248)."""
    n: int
    nr: int
    rowptr: np.ndarray  # [nr, n+1] int32
    col: np.ndarray     # [nr, 2n] int32
    val: np.ndarray     # [nr, 2n] float64
    nnz: np.ndarray     # [nr] int64

    def spmv(self, coefs, x, y=None, beta: float = 0.0) -> np.ndarray:
        c = _a(coefs, np.float64)
        x = _a(x, np.float64)
        out = np.zeros(self.n) if y is None else _a(y, np.float64).copy()
        lib().orc_spmv(self.n, self.nr, _p(self.rowptr), _p(self.col), _p(self.val), _p(c), _p(x), float(beta), _p(out))
        return out

    def abs_spmv(self, coefs, x) -> np.ndarray:
        c = _a(coefs, np.float64)
        x = _a(x, np.float64)
        out = np.zeros(self.n)
        lib().orc_abs_spmv(self.n, self.nr, _p(self.rowptr), _p(self.col), _p(self.val), _p(c), _p(x), _p(out))
        return out

    def norm1(self, coefs) -> float:
        c = _a(coefs, np.float64)
        return float(lib().orc_norm1(self.n, self.nr, _p(self.rowptr), _p(self.col), _p(self.val), _p(c)))

    def entries(self, r: int):
        """(rows, cols, vals) of A_r."""
        rp = self.rowptr[r]
        nnz = int(self.nnz[r])
        rows = np.repeat(np.arange(self.n), np.diff(rp))
        return rows, self.col[r, :nnz].copy(), self.val[r, :nnz].copy()

    def to_scipy(self, coefs):
        import scipy.sparse as sp
        A = None
        for r in range(self.nr):
            rows, cols, vals = self.entries(r)
            M = sp.csr_matrix((vals * coefs[r], (rows, cols)), shape=(self.n, self.n))
            A = M if A is None else A + M
        return A


def assemble(bounds, stoich_csr, nr: int, kind: int = PROP_TABLES, tables=None) -> CSR:
    b = _a(bounds, np.int32)
    sv, sc, sr = (_a(a, np.int32) for a in stoich_csr)
    n = num_states(b)
    rowptr = np.zeros((nr, n + 1), np.int32)
    col = np.zeros((nr, 2 * n), np.int32)
    val = np.zeros((nr, 2 * n), np.float64)
    nnz = np.zeros(nr, np.int64)
    t = _a(tables, np.float64) if tables is not None else np.zeros(1)
    rc = lib().orc_assemble_csr(len(b), nr, _p(b), _p(sv), _p(sc), _p(sr), kind, _p(t), _p(rowptr), _p(col),
                                _p(val), _p(nnz))
    if rc != 0:
        raise RuntimeError(f"orc_assemble_csr failed ({rc})")
    return CSR(n, nr, rowptr, col, val, nnz)


def assemble_model(model, kind: int = PROP_TABLES) -> CSR:
    return assemble(model.bounds, model.stoich_csr(), model.nr, kind, model.tables if kind == PROP_TABLES else None)


def propensity(kind: int, bounds, tables, x, r) -> float:
    b = _a(bounds, np.int32)
    t = _a(tables, np.float64) if tables is not None else np.zeros(1)
    xs = _a(x, np.int32)
    return float(lib().orc_propensity(kind, len(b), _p(b), _p(t), _p(xs), int(r)))


def expm(a) -> np.ndarray:
    A = np.asfortranarray(np.asarray(a, np.float64))
    F = np.empty_like(A, order="F")
    rc = lib().orc_expm(A.shape[0], _p(A), _p(F))
    if rc != 0:
        raise RuntimeError(f"orc_expm failed ({rc})")
    return F


ORC_ERR = {1: "ARG", 3: "ALLOC", 5: "NONFINITE", 6: "STEP_LIMIT"}


def expv(csr: CSR, coefs, t_final: float, v, m: int = 30, tol: float = 1e-8, iop: bool = False, q_iop: int = 2,
         anorm: float = 1.0, max_nstep: int = 10000, max_reject: int = 1000):
    """exp(t_final A) v restating KryExpvFSP::solve (src/KryExpvFSP.cu:38-188); returns (w, stats, rc)."""
    c = _a(coefs, np.float64)
    w = _a(v, np.float64).copy()
    st = ExpvStats()
    rc = lib().orc_expv(csr.n, csr.nr, _p(csr.rowptr), _p(csr.col), _p(csr.val), _p(c), float(t_final), _p(w), int(m),
                        float(tol), int(bool(iop)), int(q_iop), float(anorm), int(max_nstep), int(max_reject),
                        C.byref(st))
    return w, st.as_dict(), int(rc)


def bdf(csr: CSR, coefs, t0: float, y0, times, rtol: float = 1e-8, atol: float = 1e-12, maxl: int = 30,
        eps_lin: float = 0.005, h_init: float = 0.0, h_max: float = 0.0, max_steps: int = 10**6):
    """Variable-order BDF for dp/dt = A(t) p (bdf_oracle.c, the CVODE path of tests/test_sundials.cu:67-200).
    `coefs` is a coefficient array (time-invariant) or a callable t -> c(t).  Returns (Y [n_times, n], stats, rc)."""
    times = _a(np.atleast_1d(times), np.float64)
    y = _a(y0, np.float64)
    out = np.empty((len(times), csr.n), np.float64)
    if callable(coefs):
        nr = csr.nr

        def _tc(t, c, _user):
            v = np.asarray(coefs(t), np.float64)
            for r in range(nr):
                c[r] = float(v[r])
        cb, cp = TCOEF_FN(_tc), None
    else:
        cb, cp = TCOEF_FN(), _a(coefs, np.float64)
    st = BdfStats()
    rc = lib().orc_bdf(csr.n, csr.nr, _p(csr.rowptr), _p(csr.col), _p(csr.val), None if cp is None else _p(cp), cb,
                       None, float(t0), _p(y), _p(times), len(times), _p(out), float(rtol), float(atol), int(maxl),
                       float(eps_lin), float(h_init), float(h_max), int(max_steps), C.byref(st))
    return out, st.as_dict(), int(rc)


def bdf_change_matrix(k: int, rho: float) -> np.ndarray:
    T = np.empty((k + 1, k + 1), np.float64)
    lib().orc_bdf_change_matrix(int(k), float(rho), _p(T))
    return T


def toggle_factor_tables(bounds) -> np.ndarray:
    b = _a(bounds, np.int32)
    out = np.empty((6, int(b[0]) + int(b[1]) + 2), np.float64)
    lib().orc_toggle_factor_tables(_p(b), _p(out))
    return out


# ---- log-likelihood and its gradient (reference for the adjoint) -------------------------------
# log L(c) = sum_i sum_k D_i[k] log max(1e-44, q_i[k]), q_i = block sums of exp(t_i A(c)) p0
# (src/Likelihood.cpp:14-21 over several data times, marginalised over the fastest `block` states).

def _block_sums(p, block):
    return p.reshape(-1, block).sum(axis=1)


def loglik(csr: CSR, coefs, times, p0, counts, block: int = 1) -> float:
    """log L by scipy's expm_multiply on A(c) (FP64, exact to rounding for these sizes)."""
    from scipy.sparse.linalg import expm_multiply
    A = csr.to_scipy(np.asarray(coefs, np.float64)).tocsc()
    p, t_prev, ll = np.asarray(p0, np.float64).copy(), 0.0, 0.0
    for i, t in enumerate(times):
        if t > t_prev:
            p = expm_multiply((t - t_prev) * A, p)
        t_prev = t
        q = _block_sums(p, block)
        ll += float(np.sum(counts[i] * np.log(np.maximum(1e-44, q))))
    return ll


def loglik_grad_forward(csr: CSR, coefs, times, p0, counts, block: int = 1):
    """d log L / d log c_r by forward sensitivities: [p; s_r]' = [[A, 0], [A_r, A]] [p; s_r],
    s_r(0) = 0, so s_r(t) = d p(t) / d c_r; then d log L / d c_r = sum_i g_i^T s_r(t_i) with
    g_i = M^T (D_i / q_i).  Returns (log L, gradient wrt log c)."""
    import scipy.sparse as sp
    from scipy.sparse.linalg import expm_multiply
    c = np.asarray(coefs, np.float64)
    n, nr = csr.n, csr.nr
    A = csr.to_scipy(c)
    grads = np.zeros(nr)
    ll = loglik(csr, c, times, p0, counts, block)
    for r in range(nr):
        e = np.zeros(nr)
        e[r] = 1.0
        Ar = csr.to_scipy(e)
        Z = sp.csr_matrix((n, n))
        Aug = sp.bmat([[A, Z], [Ar, A]]).tocsc()
        y = np.concatenate([np.asarray(p0, np.float64), np.zeros(n)])
        t_prev = 0.0
        for i, t in enumerate(times):
            if t > t_prev:
                y = expm_multiply((t - t_prev) * Aug, y)
            t_prev = t
            p, s = y[:n], y[n:]
            q = _block_sums(p, block)
            gq = np.where(q > 1e-44, counts[i] / np.where(q > 1e-44, q, 1.0), 0.0)
            grads[r] += float(np.dot(np.repeat(gq, block), s))
    return ll, grads * c


def augmented_sensitivity_csr(csr: CSR, r: int) -> CSR:
    """The forward-sensitivity system of reaction r as a CSR operator over 2n states:
    [p; s_r]' = [[A, 0], [A_r, A]] [p; s_r] with A = sum_k c_k A_k, written as nr + 1 matrices:
    block-diag(A_k, A_k) with coefficient c_k, and [[0, 0], [A_r, 0]] with coefficient 1."""
    n, nr = csr.n, csr.nr
    N = 2 * n
    rowptr = np.zeros((nr + 1, N + 1), np.int32)
    col = np.zeros((nr + 1, 2 * N), np.int32)
    val = np.zeros((nr + 1, 2 * N), np.float64)
    nnz = np.zeros(nr + 1, np.int64)
    for k in range(nr):
        z = int(csr.nnz[k])
        rp = csr.rowptr[k]
        rowptr[k, :n + 1] = rp
        rowptr[k, n + 1:] = z + rp[1:]
        col[k, :z] = csr.col[k, :z]
        col[k, z:2 * z] = csr.col[k, :z] + n
        val[k, :z] = csr.val[k, :z]
        val[k, z:2 * z] = csr.val[k, :z]
        nnz[k] = 2 * z
    z = int(csr.nnz[r])
    rowptr[nr, n + 1:] = csr.rowptr[r][1:]
    col[nr, :z] = csr.col[r, :z]
    val[nr, :z] = csr.val[r, :z]
    nnz[nr] = z
    return CSR(N, nr + 1, rowptr, col, val, nnz)


def loglik_grad_forward_krylov(csr: CSR, coefs, times, p0, counts, block: int, reactions, m: int = 40,
                               tol: float = 1e-13):
    """d log L / d log c_r for the listed reactions by forward sensitivities, integrated with this
    oracle's Krylov expv (orc_expv) on the augmented system of augmented_sensitivity_csr: the
    sizes where scipy's expm_multiply takes minutes per solve.  Returns (log L, {r: gradient})."""
    c = np.asarray(coefs, np.float64)
    n = csr.n
    out, ll = {}, None
    for r in reactions:
        aug = augmented_sensitivity_csr(csr, r)
        ca = np.concatenate([c, [1.0]])
        y = np.concatenate([np.asarray(p0, np.float64), np.zeros(n)])
        t_prev, g, lsum = 0.0, 0.0, 0.0
        for i, t in enumerate(times):
            if t > t_prev:
                y, _, rc = expv(aug, ca, t - t_prev, y, m=m, tol=tol, max_nstep=10**6)
                if rc != 0:
                    raise RuntimeError(f"orc_expv failed ({rc})")
            t_prev = t
            p, s = y[:n], y[n:]
            q = _block_sums(p, block)
            gq = np.where(q > 1e-44, counts[i] / np.where(q > 1e-44, q, 1.0), 0.0)
            g += float(np.dot(np.repeat(gq, block), s))
            lsum += float(np.sum(counts[i] * np.log(np.maximum(1e-44, q))))
        out[r] = g * c[r]
        ll = lsum
    return ll, out
