"""Python mirror of the reference's solver / statistics API (cme namespace, never compiled there).

  FSPSolver      <- cme::FSPSolver   (src/FSPSolver.h:16-111)
  Likelihood     <- cme::Likelihood  (src/Likelihood.h:20-57, src/Likelihood.cpp:8-33)
  generate_data  <- cme::generate_data (src/Likelihood.cpp:35-84), seeded
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import AdaptiveStatus, ModelDesc, PROP_FACTOR_FN, SolverStatus
from .fsp import FSPMat, MatrixFormat, _ptr, _stream


class FSPSolver:
    """Advances a device probability vector through output times; reports the FSP error
    sum(p(0)) - sum(p(t)) against fsp_tol after every advance.  method="krylov" uses the Krylov
    exponential of the time-invariant generator; method="bdf" the BDF integrator (rtol, atol),
    which with coefs=None follows the generator's c_r(t)."""

    def __init__(self, A: FSPMat, p, times, fsp_tol: float = 1e-4, kry_tol: float = 1e-8, m: int = 30,
                 iop: bool = False, q_iop: int = 2, coefs=None, method: str = "krylov", rtol: float = 1e-8,
                 atol: float = 1e-12):
        self._lib = A._lib
        self.A, self.p = A, p
        self.method = method
        self.times = np.ascontiguousarray(np.asarray(times, np.float64))
        cp = None
        if coefs is not None:
            self._coefs = np.ascontiguousarray(np.asarray(coefs, np.float64))
            cp = self._coefs.ctypes.data_as(C.POINTER(C.c_double))
        self._h = C.c_void_p()
        tp = self.times.ctypes.data_as(C.POINTER(C.c_double))
        if method == "bdf":
            _lib.check(self._lib, self._lib.cufsp_solver_create_bdf(
                A.handle, tp, len(self.times), float(fsp_tol), cp, float(rtol), float(atol), C.byref(self._h)),
                "cufsp_solver_create_bdf")
        elif method == "krylov":
            _lib.check(self._lib, self._lib.cufsp_solver_create(
                A.handle, tp, len(self.times), float(fsp_tol), cp, float(kry_tol), int(m), int(bool(iop)), int(q_iop),
                C.byref(self._h)), "cufsp_solver_create")
        else:
            raise ValueError(f"unknown method {method!r}")
        self.status: dict | None = None

    def set_coefs(self, coefs) -> None:
        cp = None
        if coefs is not None:
            self._coefs = np.ascontiguousarray(np.asarray(coefs, np.float64))
            cp = self._coefs.ctypes.data_as(C.POINTER(C.c_double))
        _lib.check(self._lib, self._lib.cufsp_solver_set_coefs(self._h, cp), "cufsp_solver_set_coefs")

    def next_time(self, stream=None) -> dict:
        st = SolverStatus()
        _lib.check(self._lib, self._lib.cufsp_solver_next_time(self._h, _ptr(self.p), _stream(stream), C.byref(st)),
                   "cufsp_solver_next_time")
        self.status = st.as_dict()
        return self.status

    def solve(self, stream=None) -> dict:
        st = SolverStatus()
        _lib.check(self._lib, self._lib.cufsp_solver_solve(self._h, _ptr(self.p), _stream(stream), C.byref(st)),
                   "cufsp_solver_solve")
        self.status = st.as_dict()
        return self.status

    def reset_time(self) -> None:
        _lib.check(self._lib, self._lib.cufsp_solver_reset_time(self._h), "cufsp_solver_reset_time")

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.cufsp_solver_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _model_desc(model):
    """cufsp_model_desc of a models.CMEModel (factor tables, no time coefficients); returns the
    descriptor and the arrays it points into (keep them alive while the descriptor is used)."""
    b = np.ascontiguousarray(np.asarray(model.bounds, np.int32))
    sv, sc, sr = model.stoich_csr()
    tab = np.ascontiguousarray(model.tables, np.float64)
    d = ModelDesc()
    d.n_species, d.n_reactions = model.ns, model.nr
    d.fsp_bounds = b.ctypes.data_as(C.POINTER(C.c_int))
    d.stoich_vals = sv.ctypes.data_as(C.POINTER(C.c_int))
    d.stoich_colidxs = sc.ctypes.data_as(C.POINTER(C.c_int))
    d.stoich_rowptrs = sr.ctypes.data_as(C.POINTER(C.c_int))
    d.factor_tables = tab.ctypes.data_as(C.POINTER(C.c_double))
    return d, (b, sv, sc, sr, tab)


def generate_data(model, times, x0, n_cells: int, seed: int = 20261203, coefs=None, max_events: int = 10**8,
                  lib=None) -> np.ndarray:
    """Seeded SSA snapshots: int32 array [n_times, n_cells, n_species], an independent trajectory
    per (time, cell)."""
    import torch
    lib = lib or _lib.load()
    b = np.ascontiguousarray(np.asarray(model.bounds, np.int32))
    sv, sc, sr = model.stoich_csr()
    tab = np.ascontiguousarray(model.tables, np.float64)
    d = ModelDesc()
    d.n_species, d.n_reactions = model.ns, model.nr
    d.fsp_bounds = b.ctypes.data_as(C.POINTER(C.c_int))
    d.stoich_vals = sv.ctypes.data_as(C.POINTER(C.c_int))
    d.stoich_colidxs = sc.ctypes.data_as(C.POINTER(C.c_int))
    d.stoich_rowptrs = sr.ctypes.data_as(C.POINTER(C.c_int))
    d.factor_tables = tab.ctypes.data_as(C.POINTER(C.c_double))
    c = np.ascontiguousarray(np.asarray(model.coefs(0.0) if coefs is None else coefs, np.float64))
    x0a = np.ascontiguousarray(np.asarray(x0, np.int32))
    t = np.ascontiguousarray(np.asarray(times, np.float64))
    out = torch.empty((len(t), n_cells, model.ns), dtype=torch.int32, device="cuda")
    _lib.check(lib, lib.cufsp_ssa(C.byref(d), c.ctypes.data_as(C.POINTER(C.c_double)),
                                  x0a.ctypes.data_as(C.POINTER(C.c_int)), t.ctypes.data_as(C.POINTER(C.c_double)),
                                  len(t), int(n_cells), C.c_ulonglong(seed), int(max_events), out.data_ptr(),
                                  _stream(None)), "cufsp_ssa")
    return out.cpu().numpy()


def histograms(snapshots: np.ndarray, bounds, n_marginal: int = 0):
    """Counts per time over the species n_marginal.. (the fastest n_marginal are summed out):
    returns (counts [n_times, prod(kept b+1)] float64, outside [n_times] cells outside the box)."""
    bounds = np.asarray(bounds)
    kept = bounds[n_marginal:]
    nk = int(np.prod(kept + 1))
    T = snapshots.shape[0]
    counts = np.zeros((T, nk))
    outside = np.zeros(T, np.int64)
    for it in range(T):
        x = snapshots[it][:, n_marginal:]
        inside = np.all((x >= 0) & (x <= kept), axis=1)
        outside[it] = int((~inside).sum())
        idx = np.zeros(int(inside.sum()), np.int64)
        stride = 1
        for s in range(len(kept)):
            idx += x[inside, s].astype(np.int64) * stride
            stride *= int(kept[s]) + 1
        counts[it] = np.bincount(idx, minlength=nk)
    return counts, outside


class Likelihood:
    """log L(theta) = sum_t sum_cells log max(1e-44, p_t(cell)) with p_t from the FSP solution at the
    data times, marginalised over the n_marginal fastest species (src/Likelihood.cpp:8-33).  Cells
    outside the FSP box contribute log(1e-44).  `evaluate(coefs)` takes the reaction coefficients."""

    def __init__(self, model, times, counts, outside=None, n_marginal: int = 0, fsp_tol: float = 1e-4,
                 kry_tol: float = 1e-8, m: int = 30, fmt: MatrixFormat = MatrixFormat.KRONECKER, lib=None):
        import torch
        self.model = model
        self.times = np.asarray(times, np.float64)
        self.block = int(np.prod(np.asarray(model.bounds[:n_marginal]) + 1)) if n_marginal else 1
        self.A = FSPMat.from_model(model, fmt, lib=lib)
        self.counts = torch.as_tensor(np.ascontiguousarray(counts, np.float64), device="cuda")
        assert self.counts.shape == (len(self.times), model.n_states // self.block)
        self.outside = np.zeros(len(self.times)) if outside is None else np.asarray(outside, np.float64)
        self.p0 = torch.as_tensor(model.p0(), device="cuda")
        self.p = self.p0.clone()
        self.m, self.kry_tol = m, kry_tol
        self.solver = FSPSolver(self.A, self.p, self.times, fsp_tol, kry_tol, m, coefs=model.coefs(0.0))
        self.fsp_errors: list[float] = []

    def gradient(self, coefs=None, m: int | None = None, tol: float | None = None) -> tuple[float, np.ndarray]:
        """(log L, d log L / d log c_r) at coefs (default: the model's rates) by the adjoint method
        (cufsp_likelihood_grad).  Cells outside the box add the constant outside * log(1e-44)."""
        c = np.ascontiguousarray(np.asarray(self.model.coefs(0.0) if coefs is None else coefs, np.float64))
        t = np.ascontiguousarray(self.times)
        lib = self.A._lib
        ll = C.c_double()
        g = np.zeros(self.model.nr)
        _lib.check(lib, lib.cufsp_likelihood_grad(
            self.A.handle, c.ctypes.data_as(C.POINTER(C.c_double)), len(t), t.ctypes.data_as(C.POINTER(C.c_double)),
            self.p0.data_ptr(), self.block, self.counts.data_ptr(), int(m or self.m), float(tol or self.kry_tol),
            C.byref(ll), g.ctypes.data_as(C.POINTER(C.c_double)), _stream(None)), "cufsp_likelihood_grad")
        return ll.value + float(np.sum(self.outside)) * math.log(1e-44), g

    def gradient_batched(self, coef_sets, workers: int = 4, m: int | None = None,
                         tol: float | None = None) -> tuple[np.ndarray, np.ndarray]:
        """(log L [n_sets], d log L / d log c [n_sets, n_reactions]) for many parameter sets at once
        (cufsp_likelihood_grad_batched: `workers` concurrent adjoint solves on the GPU; on the
        131,072-state gene model 4 workers measured fastest, against 2 and 8)."""
        c = np.ascontiguousarray(np.asarray(coef_sets, np.float64).reshape(-1, self.model.nr))
        ns = c.shape[0]
        t = np.ascontiguousarray(self.times)
        lib = self.A._lib
        d, _keep = _model_desc(self.model)
        ll = np.zeros(ns)
        g = np.zeros((ns, self.model.nr))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        _lib.check(lib, lib.cufsp_likelihood_grad_batched(
            C.byref(d), ns, dp(c), len(t), dp(t), self.p0.data_ptr(), self.block, self.counts.data_ptr(),
            int(m or self.m), float(tol or self.kry_tol), int(workers), dp(ll), dp(g)), "cufsp_likelihood_grad_batched")
        return ll + float(np.sum(self.outside)) * math.log(1e-44), g

    def evaluate(self, coefs=None) -> float:
        """log L at coefs (default: the last coefficients given, initially the model's rates) in one
        call of cufsp_likelihood_eval: the Krylov solve from p0 through the data times and every time's
        term reduced on the device (Likelihood::evaluate, src/Likelihood.cpp:8-33).  The FSP error at
        the last time is kept in fsp_errors."""
        if coefs is not None:
            self.solver.set_coefs(coefs)
            self._coefs = np.ascontiguousarray(np.asarray(coefs, np.float64))
        c = getattr(self, "_coefs", None)
        if c is None:
            c = self._coefs = np.ascontiguousarray(self.model.coefs(0.0))
        t = np.ascontiguousarray(self.times)
        lib = self.A._lib
        ll, err = C.c_double(), C.c_double()
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        _lib.check(lib, lib.cufsp_likelihood_eval(
            self.A.handle, dp(c), len(t), dp(t), self.p0.data_ptr(), self.block, self.counts.data_ptr(), int(self.m),
            float(self.kry_tol), C.byref(ll), C.byref(err), _stream(None)), "cufsp_likelihood_eval")
        self.fsp_errors = [err.value]
        return ll.value + float(np.sum(self.outside)) * math.log(1e-44)


class AdaptiveFSP:
    """FSP whose box grows until the FSP error (the probability that left the box) stays within
    fsp_tol * t / t_last at every output time (cufsp_adaptive_*).  `model.factor(x, s, r)` gives the
    propensity factors for any box; the model's bounds are the initial box."""

    def __init__(self, model, max_bounds, times, fsp_tol: float = 1e-6, grow: float = 1.5, kry_tol: float = 1e-8,
                 m: int = 30, coefs=None, lib=None):
        import torch
        if model.factor is None:
            raise ValueError("AdaptiveFSP needs model.factor (propensity factors for any box)")
        self._lib = lib or _lib.load()
        self.model = model
        d, self._keep = _model_desc(model)
        d.factor_tables = None
        self._cb = PROP_FACTOR_FN(lambda x, s, r: float(model.factor(x, s, r)))
        d.prop_factor = self._cb
        mb = np.ascontiguousarray(np.asarray(max_bounds, np.int32))
        c = np.ascontiguousarray(np.asarray(model.coefs(0.0) if coefs is None else coefs, np.float64))
        t = np.ascontiguousarray(np.asarray(times, np.float64))
        self._h = C.c_void_p()
        _lib.check(self._lib, self._lib.cufsp_adaptive_create(
            C.byref(d), mb.ctypes.data_as(C.POINTER(C.c_int)), float(grow), float(fsp_tol),
            c.ctypes.data_as(C.POINTER(C.c_double)), t.ctypes.data_as(C.POINTER(C.c_double)), len(t), float(kry_tol),
            int(m), C.byref(self._h)), "cufsp_adaptive_create")
        p0 = torch.as_tensor(model.p0(), device="cuda")
        _lib.check(self._lib, self._lib.cufsp_adaptive_set_initial(self._h, p0.data_ptr(), _stream(None)),
                   "cufsp_adaptive_set_initial")
        torch.cuda.synchronize()

    def next_time(self, stream=None) -> dict:
        st = AdaptiveStatus()
        _lib.check(self._lib, self._lib.cufsp_adaptive_next_time(self._h, _stream(stream), C.byref(st)),
                   "cufsp_adaptive_next_time")
        return st.as_dict()

    def solution(self):
        """(distribution on the current box as a device tensor (a copy), bounds)."""
        import torch
        ptr = C.c_void_p()
        b = (C.c_int * self.model.ns)()
        n = C.c_int64()
        _lib.check(self._lib, self._lib.cufsp_adaptive_solution(self._h, C.byref(ptr), b, C.byref(n)),
                   "cufsp_adaptive_solution")
        out = torch.empty(n.value, dtype=torch.float64, device="cuda")
        _lib.check(self._lib, self._lib.cufsp_vec_copy(n.value, ptr.value, out.data_ptr(), _stream(None)),
                   "cufsp_vec_copy")
        torch.cuda.synchronize()
        return out, list(b)

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.cufsp_adaptive_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
