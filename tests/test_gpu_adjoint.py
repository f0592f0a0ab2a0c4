"""Adjoint gradient of the log-likelihood (cufsp_likelihood_grad) against an FP64 forward-sensitivity
reference and central finite differences on the host (gpu).  Bar: 1e-6 relative."""
import numpy as np
import pytest

import oracle
from cuda_fsp_b200 import CufspError, FSPMat, Likelihood, MatrixFormat, generate_data, histograms, models

pytestmark = pytest.mark.gpu

GRAD_RTOL = 1e-6


def rel_err(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-6 * np.max(np.abs(b)))))


def synthetic_counts(model, times, block, cells, seed):
    """Multinomial histograms of the exact marginals (a stand-in for SSA data in small checks)."""
    csr = oracle.assemble_model(model)
    from scipy.sparse.linalg import expm_multiply
    A = csr.to_scipy(model.coefs(0)).tocsc()
    rng = np.random.default_rng(seed)
    p, t_prev, out = model.p0(), 0.0, []
    for t in times:
        p = expm_multiply((t - t_prev) * A, p)
        t_prev = t
        q = np.clip(p.reshape(-1, block).sum(axis=1), 0.0, None)
        out.append(rng.multinomial(cells, q / q.sum()).astype(float))
    return np.array(out)


@pytest.mark.parametrize("case", ["gene_marginal", "mass_action_joint", "toggle_joint"])
def test_adjoint_matches_forward_sensitivity(cuda, case):
    if case == "gene_marginal":
        m = models.gene_expression((1, 1, 1, 15, 15), time_varying=False)
        times, block = np.geomspace(1.0, 60.0, 8), 8
    elif case == "mass_action_joint":
        m = models.mass_action_3(bounds=(7, 7, 5))
        times, block = np.array([0.5, 1.0, 2.0]), 1
    else:
        m = models.toggle((15, 15))
        times, block = np.array([100.0, 400.0, 1000.0]), 1
    counts = synthetic_counts(m, times, block, 1000, seed=1)
    L = Likelihood(m, times, counts, n_marginal=3 if block == 8 else 0, kry_tol=1e-10)
    ll, g = L.gradient()
    csr = oracle.assemble_model(m)
    ll_ref, g_ref = oracle.loglik_grad_forward(csr, m.coefs(0), times, m.p0(), counts, block)
    assert abs(ll - ll_ref) <= 1e-8 * abs(ll_ref)
    assert rel_err(g, g_ref) <= GRAD_RTOL, (g, g_ref)


def test_adjoint_matches_central_differences(cuda):
    """The gradient benchmark's data shape: 1,000 SSA cells at 8 log-spaced times in [1, 60], (n, c) histograms marginalised
    over the gene states; d log L / d log theta for all 12 rates against central differences
    (h = 1e-5) of the host log-likelihood."""
    m = models.gene_expression((1, 1, 1, 31, 31), time_varying=False)
    times = np.geomspace(1.0, 60.0, 8)
    snaps = generate_data(m, times, [0, 0, 0, 0, 0], 1000, seed=20261205)
    counts, outside = histograms(snaps, m.bounds, n_marginal=3)
    L = Likelihood(m, times, counts, outside=outside, n_marginal=3, kry_tol=1e-10)
    ll, g = L.gradient()
    csr = oracle.assemble_model(m)
    c0, h = m.coefs(0), 1e-5
    fd = np.zeros(m.nr)
    for r in range(m.nr):
        cp, cm = c0.copy(), c0.copy()
        cp[r] *= np.exp(h)
        cm[r] *= np.exp(-h)
        fd[r] = (oracle.loglik(csr, cp, times, m.p0(), counts, 8) - oracle.loglik(csr, cm, times, m.p0(), counts, 8)) / (2 * h)
    # central differences carry cancellation noise of order eps |log L| / h on every component, so
    # the bar is relative to the gradient's largest component
    assert np.max(np.abs(g - fd)) <= GRAD_RTOL * np.max(np.abs(fd)), (g, fd)
    ll_ref = oracle.loglik(csr, c0, times, m.p0(), counts, 8) + outside.sum() * np.log(1e-44)
    assert abs(ll - ll_ref) <= 1e-8 * abs(ll_ref)


def test_adjoint_gradient_at_other_rates(cuda):
    m = models.gene_expression((1, 1, 1, 15, 15), time_varying=False)
    times = np.array([2.0, 5.0, 20.0])
    counts = synthetic_counts(m, times, 8, 500, seed=3)
    L = Likelihood(m, times, counts, n_marginal=3, kry_tol=1e-10)
    c = m.coefs(0) * np.exp(np.random.default_rng(4).uniform(-1, 1, m.nr))
    _, g = L.gradient(c)
    _, g_ref = oracle.loglik_grad_forward(oracle.assemble_model(m), c, times, m.p0(), counts, 8)
    assert rel_err(g, g_ref) <= GRAD_RTOL


def test_adjoint_rejects_bad_requests(cuda):
    m = models.gene_expression((1, 1, 1, 7, 7), time_varying=False)
    times = np.array([1.0])
    counts = np.ones((1, m.n_states // 8))
    L = Likelihood(m, times, counts, n_marginal=3, fmt=MatrixFormat.HYB)
    with pytest.raises(CufspError) as ei:
        L.gradient()
    assert ei.value.name == "CUFSP_ERR_UNSUPPORTED"


def test_batched_gradients_equal_single_gradients(cuda):
    """cufsp_likelihood_grad_batched (concurrent workers) gives each set's single-call result."""
    m = models.gene_expression((1, 1, 1, 15, 15), time_varying=False)
    times = np.array([1.0, 4.0, 12.0])
    counts = synthetic_counts(m, times, 8, 300, seed=5)
    L = Likelihood(m, times, counts, n_marginal=3, kry_tol=1e-10)
    rng = np.random.default_rng(6)
    sets = np.stack([m.coefs(0) * np.exp(rng.uniform(-0.5, 0.5, m.nr)) for _ in range(6)])
    ll, g = L.gradient_batched(sets, workers=3)
    # Concurrent workers take the multi-launch Arnoldi pass, a single call on this size the
    # persistent one: the same arithmetic in another summation order, far inside kry_tol = 1e-10.
    for i in range(6):
        lli, gi = L.gradient(sets[i])
        assert abs(ll[i] - lli) <= 1e-11 * abs(lli)
        assert np.max(np.abs(g[i] - gi)) <= 1e-9 * np.max(np.abs(gi))


def test_torch_autograd_wrapper(cuda):
    """torch.autograd through log_likelihood gives the adjoint gradient (d log L / d log theta)."""
    import torch
    from cuda_fsp_b200.autograd import log_likelihood
    m = models.gene_expression((1, 1, 1, 15, 15), time_varying=False)
    times = np.array([2.0, 6.0])
    counts = synthetic_counts(m, times, 8, 400, seed=8)
    L = Likelihood(m, times, counts, n_marginal=3, kry_tol=1e-10)
    lt = torch.tensor(np.log(m.coefs(0)), dtype=torch.float64, requires_grad=True)
    ll = log_likelihood(lt, L)
    ll.backward()
    ll_ref, g_ref = L.gradient(np.exp(lt.detach().numpy()))  # the same rates, bit for bit
    assert abs(ll.item() - ll_ref) <= 1e-12 * abs(ll_ref)
    assert np.max(np.abs(lt.grad.numpy() - g_ref)) <= 1e-9 * np.max(np.abs(g_ref))


def test_adjoint_through_the_launch_sequence(cuda):
    """The gradient with the multi-launch Arnoldi pass (the path of generators above the persistent
    pass's size: the transposed generator action is the specialised kernel's A^T pass), run in a child
    process with CUFSP_ARNOLDI_PERSISTENT=0, against forward sensitivities."""
    import json
    import os
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    code = (
        "import json, numpy as np, sys; sys.path.insert(0, %r)\n"
        "from cuda_fsp_b200 import Likelihood, models\n"
        "m = models.gene_expression((1, 1, 1, 15, 15), time_varying=False)\n"
        "times = np.geomspace(1.0, 60.0, 8)\n"
        "counts = np.random.default_rng(1).integers(0, 4, size=(8, m.n_states // 8)).astype(float)\n"
        "L = Likelihood(m, times, counts, n_marginal=3, kry_tol=1e-10)\n"
        "ll, g = L.gradient()\n"
        "print(json.dumps({'ll': ll, 'g': list(g)}))\n" % str(root))
    env = dict(os.environ, CUFSP_ARNOLDI_PERSISTENT="0")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    m = models.gene_expression((1, 1, 1, 15, 15), time_varying=False)
    times = np.geomspace(1.0, 60.0, 8)
    counts = np.random.default_rng(1).integers(0, 4, size=(8, m.n_states // 8)).astype(float)
    ll_ref, g_ref = oracle.loglik_grad_forward(oracle.assemble_model(m), m.coefs(0), times, m.p0(), counts, 8)
    assert abs(out["ll"] - ll_ref) <= 1e-8 * abs(ll_ref)
    assert rel_err(np.array(out["g"]), g_ref) <= GRAD_RTOL, (out["g"], g_ref)
