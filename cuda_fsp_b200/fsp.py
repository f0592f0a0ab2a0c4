"""Python mirror of the reference's C++ API over the cufsp C ABI.

  FSPMat      <- cuFSP::FSPMat      (src/FSPMat.h:21-56)
  KryExpvFSP  <- cuFSP::KryExpvFSP  (src/KryExpvFSP.h:20-108)

Vectors are CUDA tensors (torch.float64, contiguous) or raw device addresses (int).  Work is
ordered on torch's current CUDA stream.  Errors raise CufspError carrying the C status.
"""
from __future__ import annotations

import ctypes as C
from enum import IntEnum
from typing import Callable

import numpy as np

from . import _lib
from ._lib import CufspError, ExpvStats, ModelDesc


class MatrixFormat(IntEnum):
    """cuFSP::MatrixFormat (src/FSPMat.h:17-19)."""
    CUDA_CSR = 0
    HYB = 1
    KRONECKER = 2


def _ptr(x) -> int:
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        import torch
        if not x.is_cuda or x.dtype != torch.float64 or not x.is_contiguous():
            raise ValueError("expected a contiguous torch.float64 CUDA tensor")
        return x.data_ptr()
    raise TypeError(f"cannot take a device address of {type(x)!r}")


def _stream(stream) -> int:
    if stream is not None:
        return int(stream)
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.current_stream().cuda_stream
    except ImportError:
        pass
    return 0


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


class FSPMat:
    """The CME generator A(t) = sum_r c_r(t) A_r on the box 0 <= x_s <= fsp_dim[s].

    stoich: (vals, col_idxs, row_ptrs) CSR with one row per reaction (the reference's CSRMatInt),
            or a dense [n_reactions, n_species] array of net changes.
    prop:   factor tables [n_reactions, sum(b_s+1)] (float64), a host factor function
            f(x, species, reaction) (the reference's PropFactorFun), or an int device address of a
            propensity __device__ function (the reference's PropFun; sparse formats only, and only
            from the same device-linked module as the library, see libcufsp_testmodels.so).
    t_func: c(t) -> array[n_reactions], or f(t, out) filling out (TcoefFun); None means c_r = 1.
    """

    def __init__(self, n_reactions: int, n_species: int, fsp_dim, stoich, t_func=None, prop=None,
                 format: MatrixFormat = MatrixFormat.CUDA_CSR, lib: C.CDLL | None = None):
        self._lib = lib or _lib.load()
        self.ns, self.nr = int(n_species), int(n_reactions)
        self.format = MatrixFormat(format)
        self.bounds = _i32(fsp_dim)
        if isinstance(stoich, tuple):
            sv, sc, sr = (_i32(a) for a in stoich)
        else:
            dense = np.asarray(stoich, np.int32).reshape(self.nr, self.ns)
            vals, cols, rows = [], [], [0]
            for r in range(self.nr):
                for s in range(self.ns):
                    if dense[r, s]:
                        vals.append(dense[r, s])
                        cols.append(s)
                rows.append(len(vals))
            sv, sc, sr = _i32(vals), _i32(cols), _i32(rows)
        self._keep = [self.bounds, sv, sc, sr]
        d = ModelDesc()
        d.n_species, d.n_reactions = self.ns, self.nr
        d.fsp_bounds = self.bounds.ctypes.data_as(C.POINTER(C.c_int))
        d.stoich_vals = sv.ctypes.data_as(C.POINTER(C.c_int))
        d.stoich_colidxs = sc.ctypes.data_as(C.POINTER(C.c_int))
        d.stoich_rowptrs = sr.ctypes.data_as(C.POINTER(C.c_int))
        if isinstance(prop, np.ndarray):
            tab = np.ascontiguousarray(prop, dtype=np.float64)
            self._keep.append(tab)
            d.factor_tables = tab.ctypes.data_as(C.POINTER(C.c_double))
        elif isinstance(prop, int):
            d.prop_device = prop
        elif callable(prop):
            cb = _lib.PROP_FACTOR_FN(lambda x, s, r: float(prop(x, s, r)))
            self._keep.append(cb)
            d.prop_factor = cb
        else:
            raise ValueError("prop must be factor tables, a factor function or a device function address")
        self._t_func = t_func
        if t_func is not None:
            nr = self.nr

            def _tc(t, out, user):
                try:
                    v = t_func(t)
                except TypeError:
                    buf = np.zeros(nr)
                    t_func(t, buf)
                    v = buf
                v = np.asarray(v, dtype=np.float64).reshape(nr)
                for r in range(nr):
                    out[r] = v[r]

            cb = _lib.TCOEF_FN(_tc)
            self._keep.append(cb)
            d.tcoef = cb
        self._h = C.c_void_p()
        _lib.check(self._lib, self._lib.cufsp_mat_create(C.byref(d), int(self.format), C.byref(self._h)),
                   "cufsp_mat_create")
        n = C.c_int64()
        self._lib.cufsp_mat_num_states(self._h, C.byref(n))
        self.n = int(n.value)

    @classmethod
    def from_model(cls, model, format: MatrixFormat = MatrixFormat.KRONECKER, prop=None, lib=None) -> "FSPMat":
        t_func = model.coefs if model.tcoef is not None else (lambda t, _r=model.rates: _r)
        return cls(model.nr, model.ns, model.bounds, model.stoich_csr(), t_func,
                   model.tables if prop is None else prop, format, lib=lib)

    # getters, src/FSPMat.cu:108-118
    def get_n_rows(self) -> int:
        return self.n

    def get_n_species(self) -> int:
        return self.ns

    def get_n_reactions(self) -> int:
        return self.nr

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def action(self, t: float, x, y, stream=None) -> None:
        """y += A(t) x  (FSPMat::action, src/FSPMat.cu:102-105)."""
        _lib.check(self._lib, self._lib.cufsp_mat_action(self._h, float(t), _ptr(x), _ptr(y), _stream(stream)),
                   "cufsp_mat_action")

    def apply(self, x, y, coefs=None, alpha: float = 1.0, beta: float = 0.0, t: float = 0.0, stream=None) -> None:
        """y = alpha * A x + beta * y with explicit coefficients (or c(t) when coefs is None)."""
        cp = None
        if coefs is not None:
            carr = np.ascontiguousarray(np.asarray(coefs, np.float64).reshape(self.nr))
            cp = carr.ctypes.data_as(C.POINTER(C.c_double))
        _lib.check(self._lib, self._lib.cufsp_mat_apply(self._h, float(t), cp, float(alpha), _ptr(x), float(beta),
                                                        _ptr(y), _stream(stream)), "cufsp_mat_apply")

    def apply_transpose(self, x, y, coefs=None, alpha: float = 1.0, t: float = 0.0, stream=None) -> None:
        """y = alpha * A^T x (KRONECKER format; the adjoint solves' operator)."""
        cp = None
        if coefs is not None:
            carr = np.ascontiguousarray(np.asarray(coefs, np.float64).reshape(self.nr))
            cp = carr.ctypes.data_as(C.POINTER(C.c_double))
        _lib.check(self._lib, self._lib.cufsp_mat_apply_transpose(self._h, float(t), cp, float(alpha), _ptr(x), _ptr(y),
                                                                  _stream(stream)), "cufsp_mat_apply_transpose")

    def action_host(self, t: float, x_host, y_host) -> None:
        """y_host += A(t) x_host on host buffers (pinned for full speed); synchronous."""
        def hp(a):
            if hasattr(a, "data_ptr"):
                return a.data_ptr()
            return a.ctypes.data
        _lib.check(self._lib, self._lib.cufsp_mat_action_host(self._h, float(t), hp(x_host), hp(y_host)),
                   "cufsp_mat_action_host")

    def watchdog(self) -> int:
        """1 if a bounded barrier wait of the TMA-fed kernel expired since the last call."""
        t = C.c_int()
        _lib.check(self._lib, self._lib.cufsp_mat_watchdog(self._h, C.byref(t)), "cufsp_mat_watchdog")
        return int(t.value)

    def describe(self) -> str:
        """The kernel that serves this generator's action (and, for KRONECKER generators that do
        not use the runtime-specialised plane kernel, why not)."""
        buf = C.create_string_buffer(1024)
        _lib.check(self._lib, self._lib.cufsp_mat_describe(self._h, buf, len(buf)), "cufsp_mat_describe")
        return buf.value.decode()

    def export_propensities(self):
        import torch
        out = torch.empty((self.nr, self.n), dtype=torch.float64, device="cuda")
        _lib.check(self._lib, self._lib.cufsp_mat_export_propensities(self._h, out.data_ptr(), _stream(None)),
                   "cufsp_mat_export_propensities")
        return out

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.cufsp_mat_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class KryExpvFSP:
    """exp(t_final A) v by the adaptive Krylov method (cuFSP::KryExpvFSP, src/KryExpvFSP.h:20-108).

    matvec: an FSPMat (evaluated with c(t_mat)), or a callable mv(x_ptr, y_ptr) that accumulates
            A x into a zeroed y (the reference's MVFun).  v: CUDA float64 tensor, updated in place.
    """

    def __init__(self, t_final: float, matvec, v, m: int = 30, tol: float = 1.0e-8, iop: bool = False,
                 q_iop: int = 2, anorm: float = 1.0, t_mat: float = 0.0, coefs=None, lib: C.CDLL | None = None):
        self._lib = lib or (matvec._lib if isinstance(matvec, FSPMat) else _lib.load())
        self.v = v
        n = v.numel() if hasattr(v, "numel") else int(len(v))
        self._h = C.c_void_p()
        _lib.check(self._lib, self._lib.cufsp_expv_create(int(n), int(m), float(tol), int(bool(iop)), int(q_iop),
                                                          float(anorm), C.byref(self._h)), "cufsp_expv_create")
        self._keep = []
        if isinstance(matvec, FSPMat):
            if coefs is not None:
                carr = np.ascontiguousarray(np.asarray(coefs, np.float64))
                _lib.check(self._lib, self._lib.cufsp_expv_bind_mat_coefs(
                    self._h, matvec.handle, carr.ctypes.data_as(C.POINTER(C.c_double))), "cufsp_expv_bind_mat")
            else:
                _lib.check(self._lib, self._lib.cufsp_expv_bind_mat(self._h, matvec.handle, float(t_mat)),
                           "cufsp_expv_bind_mat")
        elif callable(matvec):
            def _mv(x, y, user, stream):
                try:
                    matvec(int(x or 0), int(y or 0))
                    return 0
                except Exception:
                    return 1
            cb = _lib.MATVEC_FN(_mv)
            self._keep.append(cb)
            _lib.check(self._lib, self._lib.cufsp_expv_bind_matvec(self._h, cb, None), "cufsp_expv_bind_matvec")
        else:
            raise TypeError("matvec must be an FSPMat or a callable")
        self._matvec = matvec
        self.set_final_time(t_final)
        self._max_nstep, self._max_reject = 10000, 1000

    def set_final_time(self, t_final: float) -> None:
        _lib.check(self._lib, self._lib.cufsp_expv_set_final_time(self._h, float(t_final)), "cufsp_expv_set_final_time")
        self.t_final = float(t_final)

    @property
    def max_nstep(self) -> int:
        return self._max_nstep

    @max_nstep.setter
    def max_nstep(self, v: int) -> None:
        self._max_nstep = int(v)
        _lib.check(self._lib, self._lib.cufsp_expv_set_limits(self._h, self._max_nstep, self._max_reject), "set_limits")

    @property
    def max_reject(self) -> int:
        return self._max_reject

    @max_reject.setter
    def max_reject(self, v: int) -> None:
        self._max_reject = int(v)
        _lib.check(self._lib, self._lib.cufsp_expv_set_limits(self._h, self._max_nstep, self._max_reject), "set_limits")

    def solve(self, stream=None) -> dict:
        st = ExpvStats()
        _lib.check(self._lib, self._lib.cufsp_expv_solve(self._h, _ptr(self.v), _stream(stream), C.byref(st)),
                   "cufsp_expv_solve")
        return st.as_dict()

    def step(self, stream=None) -> None:
        _lib.check(self._lib, self._lib.cufsp_expv_step(self._h, _ptr(self.v), _stream(stream)), "cufsp_expv_step")

    def reset_time(self) -> None:
        _lib.check(self._lib, self._lib.cufsp_expv_reset_time(self._h), "cufsp_expv_reset_time")

    def final_time_reached(self) -> bool:
        r = C.c_int()
        _lib.check(self._lib, self._lib.cufsp_expv_final_time_reached(self._h, C.byref(r)), "final_time_reached")
        return bool(r.value)

    @property
    def stats(self) -> dict:
        st = ExpvStats()
        _lib.check(self._lib, self._lib.cufsp_expv_get_stats(self._h, C.byref(st)), "cufsp_expv_get_stats")
        return st.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.cufsp_expv_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def num_states(fsp_dim) -> int:
    """rect_fsp_num_states (src/cme_util.cu:55-62)."""
    lib = _lib.load()
    b = _i32(fsp_dim)
    n = C.c_int64()
    _lib.check(lib, lib.cufsp_num_states(len(b), b.ctypes.data_as(C.POINTER(C.c_int)), C.byref(n)), "cufsp_num_states")
    return int(n.value)


def get_states(fsp_dim, stream=None):
    """fsp_get_states (src/cme_util.cu:24-41): int32 CUDA tensor [n_states, n_species]."""
    import torch
    lib = _lib.load()
    b = _i32(fsp_dim)
    n = num_states(b)
    out = torch.empty((n, len(b)), dtype=torch.int32, device="cuda")
    _lib.check(lib, lib.cufsp_get_states(len(b), b.ctypes.data_as(C.POINTER(C.c_int)), out.data_ptr(),
                                         _stream(stream)), "cufsp_get_states")
    return out


def expm(a: np.ndarray) -> np.ndarray:
    """Pade(13,13) scaling-and-squaring exponential of a small dense matrix (host)."""
    lib = _lib.load()
    A = np.asfortranarray(np.asarray(a, np.float64))
    k = A.shape[0]
    F = np.empty_like(A, order="F")
    _lib.check(lib, lib.cufsp_expm_host(k, A.ctypes.data_as(C.POINTER(C.c_double)),
                                        F.ctypes.data_as(C.POINTER(C.c_double))), "cufsp_expm_host")
    return F


def expm_blocktri(a: np.ndarray, k1: int) -> np.ndarray:
    """exp of a block upper-triangular matrix [[A11, A12], [0, A22]] with A11 of size k1 (host; the
    lower-left block of `a` is not read): the same Pade(13,13) method with three block products per
    matrix product."""
    lib = _lib.load()
    A = np.asfortranarray(np.asarray(a, np.float64))
    k = A.shape[0]
    F = np.empty_like(A, order="F")
    _lib.check(lib, lib.cufsp_expm_blocktri_host(int(k1), k - int(k1), A.ctypes.data_as(C.POINTER(C.c_double)),
                                                 F.ctypes.data_as(C.POINTER(C.c_double))), "cufsp_expm_blocktri_host")
    return F


__all__ = ["MatrixFormat", "FSPMat", "KryExpvFSP", "CufspError", "num_states", "get_states", "expm",
           "expm_blocktri"]
