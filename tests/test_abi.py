"""The C-ABI library loads, exports every declared entry point, and its host-side logic works (CPU)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
from cuda_fsp_b200 import _lib, models
from cuda_fsp_b200.fsp import FSPMat, MatrixFormat

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        names |= set(re.findall(r"\b(cufsp_[a-z0-9_]+)\s*\(", text))
    return sorted(n for n in names if not n.endswith("_fn"))


def test_library_exports_every_declared_symbol(built):
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert set(_lib.SIGNATURES) <= set(syms)


def test_status_strings(built):
    lib = _lib.load()
    for code, name in _lib.STATUS.items():
        assert lib.cufsp_status_string(code).decode() == name


def test_host_indexing_matches_oracle(built):
    lib = _lib.load()
    for b in ([3, 4, 2], [1, 1, 1, 127, 127], [255, 255, 255]):
        ba = np.asarray(b, np.int32)
        n = C.c_int64()
        _lib.check(lib, lib.cufsp_num_states(len(b), ba.ctypes.data_as(C.POINTER(C.c_int)), C.byref(n)), "num")
        assert n.value == oracle.num_states(b)
        rng = np.random.default_rng(0)
        for i in rng.integers(0, n.value, size=50):
            s = np.empty(len(b), np.int32)
            _lib.check(lib, lib.cufsp_indx2state(int(i), s.ctypes.data_as(C.POINTER(C.c_int)), len(b),
                                                 ba.ctypes.data_as(C.POINTER(C.c_int))), "i2s")
            assert np.array_equal(s, oracle.indx2state(i, b))
            j = C.c_int64()
            _lib.check(lib, lib.cufsp_state2indx(s.ctypes.data_as(C.POINTER(C.c_int)), len(b),
                                                 ba.ctypes.data_as(C.POINTER(C.c_int)), C.byref(j)), "s2i")
            assert j.value == i


def test_host_expm_matches_oracle(built):
    import scipy.linalg as sla
    from cuda_fsp_b200 import expm
    rng = np.random.default_rng(3)
    for k, s in [(3, 0.5), (32, 2.0), (32, 40.0)]:
        A = rng.standard_normal((k, k)) * s
        E = sla.expm(A)
        assert np.abs(expm(A) - oracle.expm(A)).max() <= 1e-12 * np.abs(E).max()
        assert np.abs(expm(A) - E).max() <= 1e-12 * np.abs(E).max()


def test_host_blocktri_expm_matches_full(built):
    """The block upper-triangular exponential (the adjoint's Van Loan matrices [[tau G, tau z y^T],
    [0, tau H^T]]) equals the full one and SciPy's, for blocks that are and are not multiples of the
    8-wide padding, small and large norms; the lower-left block is never read."""
    import scipy.linalg as sla
    from cuda_fsp_b200 import CufspError
    from cuda_fsp_b200.fsp import expm, expm_blocktri
    rng = np.random.default_rng(4)
    for k1, k2, s in [(30, 30, 0.5), (29, 31, 3.0), (1, 1, 1.0), (5, 40, 0.2), (40, 3, 20.0), (8, 8, 0.0)]:
        A = rng.standard_normal((k1 + k2, k1 + k2)) * s
        A[k1:, :k1] = 0.0
        E = sla.expm(A)
        Ab = A.copy()
        Ab[k1:, :k1] = np.nan
        F = expm_blocktri(Ab, k1)
        assert np.all(F[k1:, :k1] == 0.0)
        assert np.abs(F - E).max() <= 1e-12 * np.abs(E).max()
        assert np.abs(F - expm(A)).max() <= 1e-13 * np.abs(E).max()
    with pytest.raises(CufspError) as ei:  # an empty diagonal block is an argument error
        expm_blocktri(np.eye(4), 0)
    assert ei.value.name == "CUFSP_ERR_INVALID_ARG"
    with pytest.raises(CufspError) as ei:  # NaN/Inf in the blocks that are read
        A = np.eye(6)
        A[0, 5] = np.inf
        expm_blocktri(A, 3)
    assert ei.value.name == "CUFSP_ERR_NONFINITE"


def test_invalid_models_rejected_before_any_device_work(built):
    m = models.toggle((31, 31))
    with pytest.raises(_lib.CufspError) as e:
        FSPMat(m.nr, m.ns, [70000, 70000], m.nu, prop=np.ones((6, 140002)))
    assert e.value.name == "CUFSP_ERR_OVERFLOW"
    with pytest.raises(_lib.CufspError) as e:
        FSPMat(m.nr, m.ns, [31, -1], m.nu, prop=m.tables)
    assert e.value.name == "CUFSP_ERR_INVALID_ARG"
    bad = m.tables.copy()
    bad[2, 5] = np.nan
    with pytest.raises(_lib.CufspError) as e:
        FSPMat(m.nr, m.ns, m.bounds, m.nu, prop=bad, format=MatrixFormat.KRONECKER)
    assert e.value.name == "CUFSP_ERR_NONFINITE"
    with pytest.raises(_lib.CufspError) as e:
        FSPMat(m.nr, m.ns, m.bounds, (np.array([1], np.int32), np.array([5], np.int32), np.array([0, 1, 1, 1, 1, 1, 1], np.int32)),
               prop=m.tables)
    assert e.value.name == "CUFSP_ERR_INVALID_ARG"


def test_no_device_is_an_error_not_a_fallback(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    m = models.toggle((31, 31))
    with pytest.raises(_lib.CufspError) as e:
        FSPMat(m.nr, m.ns, m.bounds, m.nu, prop=m.tables, format=MatrixFormat.KRONECKER)
    assert e.value.name == "CUFSP_ERR_NO_DEVICE"


def test_models_are_consistent():
    for m in (models.toggle(), models.birth_death_2(), models.gene_expression(), models.mass_action_3(25)):
        assert m.tables.shape == (m.nr, sum(b + 1 for b in m.bounds))
        assert np.isfinite(m.tables).all()
        assert m.coefs(3.0).shape == (m.nr,)
        p0 = m.p0()
        assert p0.shape == (m.n_states,) and abs(p0.sum() - 1.0) < 1e-6
    assert models.birth_death_2().n_states == 32768
    assert models.gene_expression().n_states == 131072
    assert models.mass_action_3().n_states == 16777216
