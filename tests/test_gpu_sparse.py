"""Sparse (CSR/HYB) format: the network-specialised kernel against the oracle and the generic kernel,
and generators built from a caller-evaluated propensity table (gpu)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from cuda_fsp_b200 import FSPMat, MatrixFormat, _lib, models
from cuda_fsp_b200.likelihood import _model_desc

pytestmark = pytest.mark.gpu

MATVEC_RTOL = 1e-13


def dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def check_against_oracle(A, m, x, y0, accumulate):
    import torch
    c = m.coefs(0)
    y = dev(y0)
    A.apply(dev(x), y, coefs=c, beta=1.0 if accumulate else 0.0)
    torch.cuda.synchronize()
    csr = oracle.assemble_model(m)
    ref = csr.spmv(c, x, y0 if accumulate else None, beta=1.0 if accumulate else 0.0)
    scale = csr.abs_spmv(c, x).max() + (np.abs(y0).max() if accumulate else 0.0)
    err = np.abs(y.cpu().numpy() - ref).max()
    assert err <= MATVEC_RTOL * scale, (m.name, m.bounds, err / scale)


@pytest.mark.parametrize("make", [
    lambda: models.mass_action_3(bounds=(63, 31, 15)),       # 3 species, even
    lambda: models.mass_action_3(bounds=(6, 9, 4)),          # tiny, odd extents, even n
    lambda: models.gene_expression((1, 1, 1, 40, 23), time_varying=False),  # 5 species
    lambda: models.toggle((31, 31)),
    lambda: models.toggle((30, 30)),                          # odd n: the generic kernel
])
def test_specialised_sparse_kernel_matches_oracle(cuda, make):
    m = make()
    A = FSPMat.from_model(m, MatrixFormat.HYB)
    if m.n_states % 2 == 0:
        assert "specialised" in A.describe()
    else:
        assert "k_sparse_mv" in A.describe()
    rng = np.random.default_rng(3)
    x = rng.uniform(0, 1, m.n_states)
    y0 = rng.uniform(-1, 1, m.n_states)
    check_against_oracle(A, m, x, y0, accumulate=True)
    check_against_oracle(A, m, x, y0, accumulate=False)


def test_specialised_equals_generic_kernel(cuda, monkeypatch):
    """Same operator from both sparse kernels, including partial ranges (the host-buffer pipeline's
    slabs start and end at odd indices)."""
    import torch
    m = models.mass_action_3(bounds=(37, 20, 11))
    A = FSPMat.from_model(m, MatrixFormat.HYB)
    monkeypatch.setenv("CUFSP_SPARSE_RTC", "0")
    G = FSPMat.from_model(m, MatrixFormat.HYB)
    monkeypatch.delenv("CUFSP_SPARSE_RTC")
    assert "specialised" in A.describe() and "k_sparse_mv" in G.describe()
    rng = np.random.default_rng(5)
    x = torch.from_numpy(rng.uniform(0, 1, m.n_states)).pin_memory()
    ya = torch.from_numpy(rng.uniform(-1, 1, m.n_states)).pin_memory()
    yg = ya.clone().pin_memory()
    A.action_host(0.0, x, ya)
    G.action_host(0.0, x, yg)
    scale = oracle.assemble_model(m).abs_spmv(m.coefs(0), x.numpy()).max()
    assert (ya - yg).abs().max().item() <= MATVEC_RTOL * scale


def test_generator_from_host_propensity_table(cuda):
    """cufsp_mat_create_table: propensities evaluated by the caller (here from the factor tables on the
    host) give the same generator as the device fill."""
    import torch
    m = models.gene_expression((1, 1, 1, 20, 17), time_varying=False)
    states = oracle.get_states(m.bounds)
    off = np.concatenate([[0], np.cumsum([b + 1 for b in m.bounds])[:-1]])
    table = np.ones((m.nr, m.n_states))
    for r in range(m.nr):
        for s in range(m.ns):
            table[r] *= m.tables[r, off[s] + states[:, s]]
    lib = _lib.load()
    d, _keep = _model_desc(m)
    h = C.c_void_p()
    t = np.ascontiguousarray(table)
    _lib.check(lib, lib.cufsp_mat_create_table(C.byref(d), _lib.FORMAT_HYB, t.ctypes.data_as(C.POINTER(C.c_double)),
                                               C.byref(h)), "cufsp_mat_create_table")
    try:
        rng = np.random.default_rng(8)
        x = dev(rng.uniform(0, 1, m.n_states))
        y1 = dev(np.zeros(m.n_states))
        c = np.ascontiguousarray(m.coefs(0))
        _lib.check(lib, lib.cufsp_mat_apply(h, 0.0, c.ctypes.data_as(C.POINTER(C.c_double)), 1.0, x.data_ptr(), 0.0,
                                            y1.data_ptr(), None), "cufsp_mat_apply")
        A = FSPMat.from_model(m, MatrixFormat.HYB)
        y2 = dev(np.zeros(m.n_states))
        A.apply(x, y2, coefs=c)
        torch.cuda.synchronize()
        scale = oracle.assemble_model(m).abs_spmv(c, x.cpu().numpy()).max()
        assert (y1 - y2).abs().max().item() <= MATVEC_RTOL * scale
        # a KRONECKER request and a NaN entry are refused
        h2 = C.c_void_p()
        assert lib.cufsp_mat_create_table(C.byref(d), _lib.FORMAT_KRONECKER, t.ctypes.data_as(C.POINTER(C.c_double)),
                                          C.byref(h2)) == 1
        bad = t.copy()
        bad[3, 7] = np.nan
        assert lib.cufsp_mat_create_table(C.byref(d), _lib.FORMAT_HYB, bad.ctypes.data_as(C.POINTER(C.c_double)),
                                          C.byref(h2)) == 5
    finally:
        lib.cufsp_mat_destroy(h)
