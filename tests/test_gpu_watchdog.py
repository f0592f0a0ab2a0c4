"""The plane kernel's bounded waits: an expired wait surfaces as an error (gpu).

CUFSP_PLANE_WAIT_TRIES=0 at generator creation compiles the plane kernel with zero tries for the
waits before each plane is computed, so every such wait gives up at once, deterministically; the
kernel then waits (with its normal bound) for the copies it already issued, records the expiry in its
watchdog word and returns.  No wait is left unbounded and no copy is left in flight, so the context
stays usable, which the last step checks.
"""
import numpy as np
import pytest

import oracle
from cuda_fsp_b200 import BDFIntegrator, CufspError, FSPMat, KryExpvFSP, MatrixFormat, models

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def starved_generator(monkeypatch, model):
    monkeypatch.setenv("CUFSP_PLANE_WAIT_TRIES", "0")
    A = FSPMat.from_model(model, MatrixFormat.KRONECKER)
    monkeypatch.delenv("CUFSP_PLANE_WAIT_TRIES")
    assert "plane kernel" in A.describe()
    return A


def test_direct_action_sets_the_watchdog(cuda, monkeypatch):
    m = models.mass_action_3(bounds=(31, 31, 31))
    A = starved_generator(monkeypatch, m)
    y = dev(np.zeros(m.n_states))
    A.action(0.0, dev(np.ones(m.n_states)), y)
    assert A.watchdog() == 1
    assert A.watchdog() == 0  # reading resets the flag


def test_drivers_return_an_error(cuda, monkeypatch):
    """The Krylov driver (above the persistent pass's size the Arnoldi matvecs are plane-kernel
    launches), the BDF integrator and the host-buffer action each report CUFSP_ERR_CUDA."""
    import torch
    m = models.mass_action_3(bounds=(127, 127, 127))
    A = starved_generator(monkeypatch, m)
    with pytest.raises(CufspError) as e:
        KryExpvFSP(0.001, A, dev(m.p0()), m=10, tol=1e-8, coefs=m.coefs(0)).solve()
    assert e.value.name == "CUFSP_ERR_CUDA" and "barrier wait" in str(e.value)
    B = BDFIntegrator(A, coefs=m.coefs(0), rtol=1e-8, atol=1e-14)
    p = dev(m.p0())
    B.init(0.0, p)
    with pytest.raises(CufspError) as e:
        B.advance(1e-4, p)
    assert e.value.name == "CUFSP_ERR_CUDA"
    xh = torch.ones(m.n_states, dtype=torch.float64).pin_memory()
    yh = torch.zeros(m.n_states, dtype=torch.float64).pin_memory()
    with pytest.raises(CufspError) as e:
        A.action_host(0.0, xh, yh)
    assert e.value.name == "CUFSP_ERR_CUDA"
    # the context is intact: a normal generator of the same network matches the oracle
    A_ok = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    xh = np.random.default_rng(0).uniform(0, 1, m.n_states)
    y = dev(np.zeros(m.n_states))
    A_ok.action(0.0, dev(xh), y)
    assert A_ok.watchdog() == 0
    csr = oracle.assemble_model(m)
    c = m.coefs(0)
    err = np.abs(y.cpu().numpy() - csr.spmv(c, xh)).max()
    assert err <= 1e-13 * csr.abs_spmv(c, xh).max()
