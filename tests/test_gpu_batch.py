"""Batched persistent Krylov solver (cufsp_batch_*) against the oracle's restatement of
KryExpvFSP::solve (src/KryExpvFSP.cu:38-188) and the single-instance GPU path (gpu)."""
import numpy as np
import pytest

import oracle
from cuda_fsp_b200 import BatchKrylov, CufspError, FSPMat, KryExpvFSP, MatrixFormat, models

pytestmark = pytest.mark.gpu


def small_gene_batch(n, seed, lo=4, hi=24):
    return models.gene_batch(n, seed=seed, lo=lo, hi=hi)


def oracle_solve(model, t, **kw):
    csr = oracle.assemble_model(model)
    w, st, rc = oracle.expv(csr, model.coefs(0), t, model.p0(), **kw)
    assert rc == 0
    return w, st


def budget(t, tol=1e-8):
    """Expokit bounds the local error per unit time (delta * tol, delta = 1.2), so two correct
    implementations that round differently may differ by up to the global budget delta * tol * t;
    results are compared with a tol = 1e-13 solution against that budget."""
    return max(1e-8, 1.2 * tol * t)


def truth(model, t):
    """exp(tA) p0 to ~1e-13: the dense exponential for small boxes (a Krylov space of m = 40 does not
    fit an 8-state box; Expokit's breakdown test at tol 1e-13 then hinges on the last bit), the
    oracle's Krylov solve at tol 1e-13 otherwise."""
    if model.n_states <= 2000:
        import scipy.linalg as sla
        A = oracle.assemble_model(model).to_scipy(model.coefs(0)).toarray()
        return sla.expm(t * A) @ model.p0()
    return oracle_solve(model, t, m=40, tol=1e-13)[0]


@pytest.mark.parametrize("shape", [(0, 0), (1, 128), (4, 256), (16, 256)])
def test_batch_matches_oracle(cuda, shape):
    """Every instance is within the Krylov tolerance (1e-8) of the oracle in 1-norm and takes about
    the oracle's number of steps: reductions in another order round differently, and the step
    control's 2-significant-digit rounding of the step size can turn that into a step or two."""
    ms = small_gene_batch(12, seed=1)
    B = BatchKrylov.from_models(ms, m=30, tol=1e-8)
    if shape != (0, 0):
        B.set_shape(*shape)
    p = B.pack([mm.p0() for mm in ms])
    stats = B.solve(10.0, p)
    out = B.unpack(p)
    for mm, w, st in zip(ms, out, stats):
        ref, st_ref = oracle_solve(mm, 10.0, m=30, tol=1e-8)
        assert st["status"] == 0 and st["t"] == 10.0
        assert np.abs(w - ref).sum() <= 1e-8, (mm.bounds, np.abs(w - ref).sum())
        assert abs(st["steps"] - st_ref["n_steps"]) <= max(2, st_ref["n_steps"] // 10)
    assert "persistent launch" in B.describe()


def test_batch_matches_single_instance_path(cuda):
    import torch
    ms = small_gene_batch(6, seed=2, lo=20, hi=60)
    B = BatchKrylov.from_models(ms, m=30, tol=1e-8)
    p = B.pack([mm.p0() for mm in ms])
    B.solve(30.0, p)
    out = B.unpack(p)
    for mm, w in zip(ms, out):
        A = FSPMat.from_model(mm, MatrixFormat.KRONECKER)
        v = torch.as_tensor(mm.p0(), device="cuda")
        KryExpvFSP(30.0, A, v, m=30, tol=1e-8, coefs=mm.coefs(0)).solve()
        ref = truth(mm, 30.0)
        assert np.abs(w - ref).sum() <= budget(30.0)
        assert np.abs(v.cpu().numpy() - ref).sum() <= budget(30.0)


def test_batch_uneven_sizes_and_other_networks(cuda):
    """Instances from a few states (fewer than one warp per CTA) to thousands; a 2-species and a
    3-species network; table, identity and constant factors."""
    cases = [(models.toggle, [(1, 2), (7, 3), (40, 31), (15, 60)], 200.0),
             (lambda b: models.mass_action_3(bounds=b), [(1, 1, 1), (5, 2, 7), (12, 9, 20), (3, 30, 4)], 2.0)]
    for make, bounds, t in cases:
        ms = [make(b) for b in bounds]
        B = BatchKrylov.from_models(ms, m=20, tol=1e-8)
        p = B.pack([mm.p0() for mm in ms])
        B.solve(t, p)
        for mm, w in zip(ms, B.unpack(p)):
            err = np.abs(w - truth(mm, t)).sum()
            assert err <= budget(t), (mm.name, mm.bounds, err)


def test_batch_iop(cuda):
    """Incomplete orthogonalisation (q = 2) follows the oracle's IOP restatement."""
    ms = small_gene_batch(5, seed=3)
    B = BatchKrylov.from_models(ms, m=30, tol=1e-8, iop=True, q_iop=2)
    p = B.pack([mm.p0() for mm in ms])
    B.solve(10.0, p)
    for mm, w in zip(ms, B.unpack(p)):
        ref, _ = oracle_solve(mm, 10.0, m=30, tol=1e-8, iop=True, q_iop=2)
        assert np.abs(w - ref).sum() <= 1e-8 or np.abs(w - truth(mm, 10.0)).sum() <= budget(10.0)


def test_batch_zero_vector_and_repeat(cuda):
    """A zero vector stays zero; solving twice from the same data gives bit-identical results
    (fixed reduction order, graph replay)."""
    ms = small_gene_batch(4, seed=4)
    B = BatchKrylov.from_models(ms, m=30, tol=1e-8)
    vecs = [mm.p0() for mm in ms]
    vecs[1] = np.zeros_like(vecs[1])
    p1 = B.pack(vecs)
    p2 = B.pack(vecs)
    B.solve(5.0, p1)
    B.solve(5.0, p2)
    a, b = B.unpack(p1), B.unpack(p2)
    assert not a[1].any()
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_batch_step_limit_reports_error(cuda):
    ms = small_gene_batch(3, seed=5)
    B = BatchKrylov.from_models(ms, m=10, tol=1e-12)
    B.set_limits(1, 1000)
    p = B.pack([mm.p0() for mm in ms])
    with pytest.raises(CufspError) as ei:
        B.solve(60.0, p)
    assert ei.value.name == "CUFSP_ERR_STEP_LIMIT"
    stats = B.solve(60.0, B.pack([mm.p0() for mm in ms]), check=False)
    assert all(s["status"] == 1 for s in stats)


def test_batch_set_coefs(cuda):
    """New rate coefficients take effect at the next solve."""
    ms = small_gene_batch(4, seed=6)
    B = BatchKrylov.from_models(ms, m=30, tol=1e-8)
    ms2 = small_gene_batch(4, seed=7)
    for a, b in zip(ms, ms2):  # same boxes, other rates
        b.bounds = a.bounds
        b.tables = a.tables
    B.set_coefs(np.stack([mm.coefs(0) for mm in ms2]))
    p = B.pack([mm.p0() for mm in ms])
    B.solve(5.0, p)
    for mm, w in zip(ms2, B.unpack(p)):
        ref, _ = oracle_solve(mm, 5.0, m=30, tol=1e-8)
        assert np.abs(w - ref).sum() <= 1e-8
