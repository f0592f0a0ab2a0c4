"""FSPSolver, the log-likelihood reduction, the SSA data generator and Likelihood on the GPU,
against the oracle (gpu)."""
import math

import numpy as np
import pytest

import oracle
from cuda_fsp_b200 import FSPMat, FSPSolver, Likelihood, MatrixFormat, generate_data, histograms, models

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def oracle_path(model, coefs, times):
    """p(t_k) for each output time by successive oracle Krylov solves."""
    csr = oracle.assemble_model(model)
    p, t0, out = model.p0(), 0.0, []
    for t in times:
        p, st, rc = oracle.expv(csr, coefs, t - t0, p, m=30, tol=1e-8)
        assert rc == 0
        out.append(p.copy())
        t0 = t
    return out


def test_loglik_reduction_matches_numpy(cuda):
    import ctypes as C
    import torch
    from cuda_fsp_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(3)
    for n, block in ((1000, 1), (8192, 8), (131072, 8)):
        p = rng.uniform(0, 1e-3, n)
        p[rng.integers(0, n, 50)] = 0.0  # exercise the 1e-44 floor
        counts = rng.integers(0, 5, n // block).astype(np.float64)
        out = C.c_double()
        dp, dc = dev(p), dev(counts)  # keep the tensors alive while the kernel reads them
        _lib.check(lib, lib.cufsp_loglik(n, dp.data_ptr(), block, dc.data_ptr(), C.byref(out), None), "loglik")
        q = p.reshape(-1, block).sum(axis=1)
        ref = float(np.sum(counts * np.log(np.maximum(1e-44, q))))
        assert abs(out.value - ref) <= 1e-12 * np.sum(counts * np.abs(np.log(np.maximum(1e-44, q))))


def test_solver_steps_through_output_times(cuda):
    m = models.birth_death_2()
    times = [1.0, 2.5, 10.0]
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    p = dev(m.p0())
    S = FSPSolver(A, p, times, fsp_tol=1e-6, coefs=m.coefs(0))
    ref = oracle_path(m, m.coefs(0), times)
    for k, t in enumerate(times):
        st = S.next_time()
        assert st["time_index"] == k and st["t"] == t
        got = p.cpu().numpy()
        assert np.abs(got - ref[k]).sum() <= 1e-8
        assert abs(st["fsp_error"] - (1.0 - ref[k].sum())) <= 1e-10
        assert st["fsp_tol_exceeded"] == int(st["fsp_error"] > 1e-6)
    # reset_time keeps the vector; solve() goes straight to the last time
    p.copy_(dev(m.p0()))
    S.reset_time()
    st = S.solve()
    assert st["t"] == 10.0 and np.abs(p.cpu().numpy() - ref[-1]).sum() <= 1e-8


def test_solver_reports_truncation_error(cuda):
    """A box too small for the dynamics loses probability through the boundary outflow."""
    m = models.mass_action((10, 10), [[1, 0], [-1, 0], [0, 1], [0, -1]], [[0, 0], [1, 0], [1, 0], [0, 1]],
                           [10.0, 1.0, 0.5, 0.2])
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    p = dev(m.p0())
    S = FSPSolver(A, p, [5.0], fsp_tol=1e-3, coefs=m.coefs(0))
    st = S.next_time()
    ref = oracle_path(m, m.coefs(0), [5.0])[0]
    assert st["fsp_error"] > 0.1 and st["fsp_tol_exceeded"] == 1
    assert abs(st["fsp_error"] - (1.0 - ref.sum())) <= 1e-9


def test_ssa_reproducible_and_matches_fsp_moments(cuda):
    m = models.birth_death_2()
    times = [2.0, 10.0]
    d1 = generate_data(m, times, [0, 0], 40000, seed=11)
    d2 = generate_data(m, times, [0, 0], 40000, seed=11)
    d3 = generate_data(m, times, [0, 0], 40000, seed=12)
    assert d1.shape == (2, 40000, 2)
    assert np.array_equal(d1, d2) and not np.array_equal(d1, d3)
    ref = oracle_path(m, m.coefs(0), times)
    for k in range(len(times)):
        P = ref[k].reshape(256, 128)  # [x2][x1]
        for s, marg in ((0, P.sum(axis=0)), (1, P.sum(axis=1))):
            xs = np.arange(len(marg))
            mu = float((xs * marg).sum())
            var = float(((xs - mu) ** 2 * marg).sum())
            emp = d1[k, :, s]
            assert abs(emp.mean() - mu) <= 5.0 * math.sqrt(var / emp.size)
            # two-sided Kolmogorov distance against the FSP marginal (alpha ~ 1e-3)
            cdf = np.cumsum(marg)
            ecdf = np.searchsorted(np.sort(emp), xs, side="right") / emp.size
            assert np.abs(ecdf - cdf).max() <= 1.95 / math.sqrt(emp.size)


def test_likelihood_matches_oracle_pipeline(cuda):
    """Gene-expression model on a 2x2x2x32x32 box, data binned over (n, c) and marginalised over
    the three gene states (src/Likelihood.cpp:8-33 with marginalisation)."""
    m = models.gene_expression((1, 1, 1, 31, 31), time_varying=False)
    times = np.array([1.0, 3.0, 8.0, 20.0])
    data = generate_data(m, times, [0, 0, 0, 0, 0], 1000, seed=5)
    counts, outside = histograms(data, m.bounds, n_marginal=3)
    L = Likelihood(m, times, counts, outside, n_marginal=3)
    for scale in (1.0, 1.7):
        c = m.coefs(0) * np.where(np.arange(m.nr) % 2 == 0, scale, 1.0)
        got = L.evaluate(c)
        ref = 0.0
        for k, p in enumerate(oracle_path(m, c, times)):
            q = p.reshape(-1, 8).sum(axis=1)
            ref += float(np.sum(counts[k] * np.log(np.maximum(1e-44, q)))) + outside[k] * math.log(1e-44)
        assert abs(got - ref) <= 1e-7 * abs(ref), (got, ref)
