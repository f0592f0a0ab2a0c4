"""The two forms of the Arnoldi pass agree (gpu).

Generators up to 2^20 states run each Krylov step's Arnoldi pass as one persistent cooperative launch
(cufsp_arnoldi.cu); larger ones, and threads of the many-worker batched gradient, use the sequence of
generator / multi-dot / update launches replayed from a CUDA graph (cufsp_krylov.cu).  The two are the
same arithmetic in another summation order.  CUFSP_ARNOLDI_PERSISTENT=0 forces the launch sequence;
it is read once per process, so the reference results come from a child process.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle
from cuda_fsp_b200 import FSPMat, KryExpvFSP, Likelihood, MatrixFormat, models

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent

# Each case: (name, model factory source, format, t_final, Krylov options).
CASES = [
    ("bd2", "models.birth_death_2()", "KRONECKER", 10.0, dict(m=30, tol=1e-8)),
    ("gene_hyb", "models.gene_expression((1, 1, 1, 40, 30), time_varying=False)", "HYB", 20.0, dict(m=30, tol=1e-8)),
    ("toggle_iop", "models.toggle((60, 60))", "KRONECKER", 500.0, dict(m=20, tol=1e-8, iop=True, q_iop=2)),
    ("ma3_m7", "models.mass_action_3(bounds=(20, 17, 13))", "KRONECKER", 0.5, dict(m=7, tol=1e-8)),
    ("tiny", "models.toggle((2, 3))", "KRONECKER", 5.0, dict(m=30, tol=1e-8)),
]

_CHILD = r"""
import json, sys
import numpy as np, torch
from cuda_fsp_b200 import FSPMat, KryExpvFSP, Likelihood, MatrixFormat, models
out = {}
for name, src, fmt, t, kw in json.loads(sys.argv[1]):
    m = eval(src)
    A = FSPMat.from_model(m, getattr(MatrixFormat, fmt))
    v = torch.as_tensor(m.p0(), device="cuda")
    st = KryExpvFSP(t, A, v, coefs=m.coefs(0), **kw).solve()
    out[name] = {"v": v.cpu().numpy().tolist(), "steps": st["n_steps"]}
m = models.gene_expression((1, 1, 1, 15, 15), time_varying=False)
times = np.array([1.0, 4.0, 12.0])
counts = np.asarray(json.loads(sys.argv[2]))
L = Likelihood(m, times, counts, n_marginal=3, kry_tol=1e-10)
ll, g = L.gradient()
out["grad"] = {"ll": ll, "g": g.tolist()}
print(json.dumps(out))
"""


def _counts(model, times, block=8, cells=300):
    """Multinomial histograms of the exact marginals over the gene states."""
    from scipy.sparse.linalg import expm_multiply
    A = oracle.assemble_model(model).to_scipy(model.coefs(0)).tocsc()
    rng = np.random.default_rng(5)
    p, t_prev, out = model.p0(), 0.0, []
    for t in times:
        p = expm_multiply((t - t_prev) * A, p)
        t_prev = t
        q = np.clip(p.reshape(-1, block).sum(axis=1), 0.0, None)
        out.append(rng.multinomial(cells, q / q.sum()).astype(float))
    return np.array(out)


def test_persistent_pass_matches_launch_sequence(cuda):
    import torch
    m_g = models.gene_expression((1, 1, 1, 15, 15), time_varying=False)
    times = np.array([1.0, 4.0, 12.0])
    counts = _counts(m_g, times)
    env = dict(os.environ, CUFSP_ARNOLDI_PERSISTENT="0", PYTHONPATH=str(ROOT))
    res = subprocess.run([sys.executable, "-c", _CHILD, json.dumps(CASES), json.dumps(counts.tolist())],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    ref = json.loads(res.stdout.strip().splitlines()[-1])
    for name, src, fmt, t, kw in CASES:
        m = eval(src)
        A = FSPMat.from_model(m, getattr(MatrixFormat, fmt))
        v = torch.as_tensor(m.p0(), device="cuda")
        st = KryExpvFSP(t, A, v, coefs=m.coefs(0), **kw).solve()
        got = v.cpu().numpy()
        want = np.asarray(ref[name]["v"])
        # both are within Expokit's global error budget delta * tol * t of the exact solution
        assert np.abs(got - want).sum() <= 2.4 * kw["tol"] * max(t, 1.0), name
        assert abs(st["n_steps"] - ref[name]["steps"]) <= max(2, ref[name]["steps"] // 10), name
        # and the persistent form follows the oracle's restatement on the small cases
        if m.n_states <= 40000:
            w, _, rc = oracle.expv(oracle.assemble_model(m), m.coefs(0), t, m.p0(), **kw)
            assert rc == 0
            assert np.abs(got - w).sum() <= 2.4 * kw["tol"] * max(t, 1.0), name
    L = Likelihood(m_g, times, counts, n_marginal=3, kry_tol=1e-10)
    ll, g = L.gradient()
    g_ref = np.asarray(ref["grad"]["g"])
    assert abs(ll - ref["grad"]["ll"]) <= 1e-11 * abs(ll)
    assert np.max(np.abs(g - g_ref)) <= 1e-9 * np.max(np.abs(g_ref))


def test_persistent_pass_zero_and_breakdown(cuda):
    """A zero vector comes back unchanged; a generator without reactions that leave p0's state
    (happy breakdown at the first iteration) leaves p0 as it is."""
    import torch
    m = models.birth_death_2()
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    v = torch.zeros(m.n_states, dtype=torch.float64, device="cuda")
    KryExpvFSP(1.0, A, v, coefs=m.coefs(0)).solve()
    assert float(v.abs().max()) == 0.0
    v = torch.as_tensor(m.p0(), device="cuda")
    st = KryExpvFSP(3.0, A, v, coefs=np.zeros(m.nr)).solve()
    assert np.allclose(v.cpu().numpy(), m.p0(), rtol=1e-15, atol=0.0)
    assert st["t_now"] == 3.0
