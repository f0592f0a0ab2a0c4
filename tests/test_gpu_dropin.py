"""The C++ drop-in layer (include/cufsp.hpp) used the way the reference's own tests use the
reference API: device PropFun via cudaMemcpyFromSymbol, thrust vectors, MVFun lambda (gpu)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from cuda_fsp_b200 import generate_data, histograms, models

pytestmark = pytest.mark.gpu

EXE = Path(__file__).resolve().parent / "cpp" / "test_dropin"


def test_cpp_dropin_program(cuda, built):
    assert EXE.exists(), "tests/cpp/test_dropin is built by python -m cuda_fsp_b200.build"
    r = subprocess.run([str(EXE)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok (0 failures)" in r.stdout


def test_cpp_cme_likelihood_against_oracle(cuda, built):
    """cme::Likelihood::evaluate and ::gradient of the drop-in program (gene network, box 1x1x1x31x31,
    500 seeded-SSA cells at t = 1, 3, 8, full joint states) against the oracle: log L to 1e-8 relative,
    the gradient (d log L / d rate) against forward sensitivities to 1e-6 relative."""
    r = subprocess.run([str(EXE)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = {ln.split()[1]: ln.split()[2:] for ln in r.stdout.splitlines() if ln.startswith("CME ")}
    ll_cpp = float(lines["logL"][0])
    g_cpp = np.array([float(v) for v in lines["grad"]])
    rates = np.array([0.05, 0.04, 0.03, 2.0, 2.0, 3.0, 0.5, 1.5, 2.0, 0.5, 0.1, 0.05])
    m = models.gene_expression((1, 1, 1, 31, 31), time_varying=False)
    m.rates = rates.copy()  # the program's parameters, bit for bit
    times = np.array([1.0, 3.0, 8.0])
    snaps = generate_data(m, times, [0, 0, 0, 0, 0], 500, seed=777)
    counts, outside = histograms(snaps, m.bounds, n_marginal=0)
    csr = oracle.assemble_model(m)
    ll_ref, g_ref = oracle.loglik_grad_forward_krylov(csr, m.coefs(0), times, m.p0(), counts, 1, range(m.nr), m=40,
                                                      tol=1e-12)
    ll_ref += outside.sum() * np.log(1e-44)
    assert abs(ll_cpp - ll_ref) <= 1e-8 * abs(ll_ref), (ll_cpp, ll_ref)
    g_ref = np.array([g_ref[r] for r in range(m.nr)]) / m.coefs(0)  # d log L / d c_r
    err = np.max(np.abs(g_cpp - g_ref)) / np.max(np.abs(g_ref))
    assert err <= 1e-6, (g_cpp, g_ref)
