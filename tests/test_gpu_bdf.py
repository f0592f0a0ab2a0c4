"""BDF integrator for time-varying generators (the reference's CVODE path,
tests/test_sundials.cu:67-200) on the GPU, against the oracle's BDF and Krylov (gpu)."""
import numpy as np
import pytest

import oracle
from cuda_fsp_b200 import BDFIntegrator, CufspError, FSPMat, FSPSolver, MatrixFormat, models

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def gpu_path(model, times, fmt=MatrixFormat.KRONECKER, coefs=None, **kw):
    A = FSPMat.from_model(model, fmt)
    B = BDFIntegrator(A, coefs=coefs, **kw)
    p = dev(model.p0())
    B.init(0.0, p)
    out = []
    for t in times:
        assert B.advance(t, p) == t
        out.append(p.cpu().numpy().copy())
    return out, B.stats


@pytest.mark.parametrize("fmt", [MatrixFormat.KRONECKER, MatrixFormat.HYB])
def test_bdf_time_varying_toggle_matches_oracle(cuda, fmt):
    """tests/test_sundials.cu:55-64 coefficients on a 32^2 box."""
    m = models.toggle((31, 31), time_varying=True)
    times = [50.0, 500.0, 3000.0]
    got, st = gpu_path(m, times, fmt, rtol=1e-8, atol=1e-14)
    ref, rst, rc = oracle.bdf(oracle.assemble_model(m), m.coefs, 0.0, m.p0(), times, rtol=1e-8, atol=1e-14)
    assert rc == 0
    for k in range(len(times)):
        assert np.abs(got[k] - ref[k]).sum() <= 1e-7, k
    # same method, same decisions: step counts agree up to threshold effects
    assert abs(st["n_steps"] - rst["n_steps"]) <= max(3, rst["n_steps"] // 20), (st, rst)
    tight, _, rc = oracle.bdf(oracle.assemble_model(m), m.coefs, 0.0, m.p0(), times, rtol=1e-11, atol=1e-16)
    assert np.abs(got[-1] - tight[-1]).sum() <= 1e-6


def test_bdf_time_invariant_matches_krylov(cuda):
    m = models.birth_death_2()
    got, st = gpu_path(m, [1.0, 10.0], coefs=m.coefs(0), rtol=1e-8, atol=1e-14)
    A = oracle.assemble_model(m)
    for t, g in zip((1.0, 10.0), got):
        ref, _, rc = oracle.expv(A, m.coefs(0), t, m.p0(), tol=1e-13)
        assert np.abs(g - ref).sum() <= 1e-7
    assert st["order"] >= 3 and st["n_lin_fail"] == 0


def test_bdf_gene_expression_time_varying(cuda):
    """Gene-state x mRNA model with the switching rate k0 sigmoid((t-5)/0.5) on a 2x2x2x32x32 box,
    against the oracle; mass is conserved to the FSP truncation (test_sundials.cu:192 asserts
    |1 - sum p| <= 1e-10 on a box that loses nothing)."""
    m = models.gene_expression((1, 1, 1, 31, 31), time_varying=True)
    times = [2.0, 6.0, 20.0]
    got, st = gpu_path(m, times, rtol=1e-8, atol=1e-14)
    ref, rst, rc = oracle.bdf(oracle.assemble_model(m), m.coefs, 0.0, m.p0(), times, rtol=1e-8, atol=1e-14)
    assert rc == 0
    for k in range(len(times)):
        assert np.abs(got[k] - ref[k]).sum() <= 1e-7
        assert abs(got[k].sum() - ref[k].sum()) <= 1e-10


def test_bdf_one_step_matches_advance(cuda):
    m = models.toggle((31, 31), time_varying=True)
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    B = BDFIntegrator(A, rtol=1e-8, atol=1e-14)
    p = dev(m.p0())
    B.init(0.0, p)
    ts, t = [], 0.0
    while t < 400.0:
        t = B.step(400.0, p)
        ts.append(t)
    assert ts == sorted(ts) and ts[-1] == 400.0 and B.stats["n_steps"] == len(ts)
    one = p.cpu().numpy()
    got, _ = gpu_path(m, [400.0], rtol=1e-8, atol=1e-14)
    assert np.abs(one - got[0]).max() == 0.0


def test_solver_bdf_time_varying(cuda):
    m = models.gene_expression((1, 1, 1, 31, 31), time_varying=True)
    times = [1.0, 5.0, 10.0]
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    p = dev(m.p0())
    S = FSPSolver(A, p, times, fsp_tol=1e-6, method="bdf", rtol=1e-8, atol=1e-14)
    ref, _, rc = oracle.bdf(oracle.assemble_model(m), m.coefs, 0.0, m.p0(), times, rtol=1e-8, atol=1e-14)
    for k, t in enumerate(times):
        st = S.next_time()
        assert st["t"] == t and st["time_index"] == k
        assert np.abs(p.cpu().numpy() - ref[k]).sum() <= 1e-7
        assert abs(st["fsp_error"] - (1.0 - ref[k].sum())) <= 1e-10
    # reset_time restarts from the caller's vector
    p.copy_(dev(m.p0()))
    S.reset_time()
    st = S.solve()
    assert st["t"] == 10.0 and np.abs(p.cpu().numpy() - ref[-1]).sum() <= 1e-7


def test_bdf_errors(cuda):
    m = models.birth_death_2()
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    p = dev(m.p0())
    B = BDFIntegrator(A, coefs=m.coefs(0), max_steps=3)
    with pytest.raises(CufspError):  # advance before init
        B.advance(1.0, p)
    B.init(0.0, p)
    with pytest.raises(CufspError) as e:
        B.advance(10.0, p)
    assert "STEP_LIMIT" in str(e.value)
    B2 = BDFIntegrator(A, coefs=m.coefs(0))
    bad = dev(m.p0())
    bad[5] = float("nan")
    B2.init(0.0, bad)
    with pytest.raises(CufspError) as e:
        B2.advance(1.0, bad)
    assert "NONFINITE" in str(e.value)
    with pytest.raises(CufspError):
        BDFIntegrator(A, coefs=m.coefs(0), maxl=61)
