"""Python mirror of the time-varying integration path: the reference drives SUNDIALS CVODE (BDF,
Newton, matrix-free SPBCGS) with RHS f(t, u) = A(t) u through FSPMat::action
(tests/test_sundials.cu:67-200, problems/hog1p_5species.cu:203-336).  Here the integrator is the
library's own device BDF (cufsp_bdf_*).

    B = BDFIntegrator(A, rtol=1e-8, atol=1e-12)   # coefs=None: A's c_r(t)
    B.init(0.0, p)                                 # CVodeInit(cvode_rhs, 0, p0)
    t = B.step(t_final, p)                         # CVode(..., CV_ONE_STEP)
    B.advance(t_out, p)                            # CVode(..., CV_NORMAL) with tstop = t_out
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import BdfStats
from .fsp import FSPMat, _ptr, _stream


class BDFIntegrator:
    def __init__(self, A: FSPMat, coefs=None, rtol: float = 1e-8, atol: float = 1e-12, maxl: int = 30,
                 eps_lin: float = 0.005, h_init: float = 0.0, h_max: float = 0.0, max_steps: int = 10**6):
        self._lib = A._lib
        self.A = A
        cp = None
        if coefs is not None:
            self._coefs = np.ascontiguousarray(np.asarray(coefs, np.float64))
            cp = self._coefs.ctypes.data_as(C.POINTER(C.c_double))
        self._h = C.c_void_p()
        _lib.check(self._lib, self._lib.cufsp_bdf_create(A.handle, cp, float(rtol), float(atol), int(maxl),
                                                         C.byref(self._h)), "cufsp_bdf_create")
        _lib.check(self._lib, self._lib.cufsp_bdf_set_options(self._h, float(eps_lin), float(h_init), float(h_max),
                                                              int(max_steps)), "cufsp_bdf_set_options")

    def set_coefs(self, coefs) -> None:
        cp = None
        if coefs is not None:
            self._coefs = np.ascontiguousarray(np.asarray(coefs, np.float64))
            cp = self._coefs.ctypes.data_as(C.POINTER(C.c_double))
        _lib.check(self._lib, self._lib.cufsp_bdf_set_coefs(self._h, cp), "cufsp_bdf_set_coefs")

    def init(self, t0: float, p0, stream=None) -> None:
        _lib.check(self._lib, self._lib.cufsp_bdf_init(self._h, float(t0), _ptr(p0), _stream(stream)), "cufsp_bdf_init")

    def _advance(self, t_out, p, one_step, stream) -> float:
        tr = C.c_double()
        _lib.check(self._lib, self._lib.cufsp_bdf_advance(self._h, float(t_out), _ptr(p), int(one_step),
                                                          _stream(stream), C.byref(tr)), "cufsp_bdf_advance")
        return tr.value

    def advance(self, t_out: float, p, stream=None) -> float:
        """Integrate to t_out exactly; p receives p(t_out)."""
        return self._advance(t_out, p, 0, stream)

    def step(self, t_out: float, p, stream=None) -> float:
        """One internal step toward t_out (never past it); p receives the solution, returns its time."""
        return self._advance(t_out, p, 1, stream)

    @property
    def stats(self) -> dict:
        st = BdfStats()
        _lib.check(self._lib, self._lib.cufsp_bdf_get_stats(self._h, C.byref(st)), "cufsp_bdf_get_stats")
        return st.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.cufsp_bdf_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
