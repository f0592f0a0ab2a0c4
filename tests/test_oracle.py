"""The FP64 host oracle, pinned against the reference's own code and its known-answer tests (CPU)."""
import numpy as np
import pytest

import oracle
from conftest import require_ref
from cuda_fsp_b200 import models


def test_enumeration_known_answer():
    """tests/test_fsp_get_states.cu:21-54: bounds (1023, 1023, 3), species 0 fastest, bit-exact."""
    b = [1023, 1023, 3]
    st = oracle.get_states(b)
    assert st.shape == (1024 * 1024 * 4, 3)
    x2, x1, x0 = np.meshgrid(np.arange(4), np.arange(1024), np.arange(1024), indexing="ij")
    expect = np.stack([x0.ravel(), x1.ravel(), x2.ravel()], axis=1).astype(np.int32)
    assert np.array_equal(st, expect)


@pytest.mark.parametrize("bounds", [[3, 4, 2], [0, 5], [7], [1, 1, 1, 127, 127], [30, 2, 0, 4]])
def test_indexing_matches_reference_host_code(bounds):
    """indx2state / state2indx / rect_fsp_num_states (src/cme_util.cu:5-22,55-62) run from the
    reference's own compiled objects, against the restatement."""
    R = require_ref()
    b = np.asarray(bounds, np.int32)
    n = oracle.num_states(b)
    assert R.ref_num_states(len(b), b.ctypes.data) == n
    st = oracle.get_states(b)
    rng = np.random.default_rng(1)
    idx = np.unique(np.concatenate([[0, n - 1], rng.integers(0, n, size=min(n, 500))]))
    for i in idx:
        s = np.empty(len(b), np.int32)
        R.ref_indx2state(int(i), s.ctypes.data, len(b), b.ctypes.data)
        assert np.array_equal(s, st[i])
        assert R.ref_state2indx(s.ctypes.data, len(b), b.ctypes.data) == i
        assert oracle.state2indx(s, b) == i


def test_oracle_matches_committed_reference_vectors():
    """The same pins as the two tests around this one, against vectors the reference's own host code
    produced (tests/golden/reference_host.npz, written by tests/golden/make_reference_vectors.py
    through the compiled shim), so that they hold where the shim cannot be built."""
    from pathlib import Path
    import sys
    sys.path.insert(0, str(Path(__file__).parent / "golden"))
    from make_reference_vectors import BOUNDS, golden_models
    g = np.load(Path(__file__).parent / "golden" / "reference_host.npz")
    for k, bounds in enumerate(BOUNDS):
        b = np.asarray(bounds, np.int32)
        assert np.array_equal(g[f"box{k}_bounds"], b)
        assert oracle.num_states(b) == int(g[f"box{k}_n"])
        idx = g[f"box{k}_idx"]
        st = oracle.get_states(b)
        assert np.array_equal(st[idx], g[f"box{k}_states"])
        assert np.array_equal(g[f"box{k}_state2indx"], idx)
        assert all(oracle.state2indx(s, b) == i for s, i in zip(g[f"box{k}_states"], idx))
    for name, m in golden_models().items():
        assert np.array_equal(g[f"{name}_vals"], m.tables), name
        assert np.array_equal(g[f"{name}_offsets"], -m.nu), name


def test_factor_table_layout_matches_reference():
    """fspmat_sdkron_fill_host_data (src/fspmat_kron_kernels.cu:170-190) fills the same table
    layout the product consumes, and its offsets are -nu."""
    R = require_ref()
    for m in (models.toggle((31, 31)), models.gene_expression((1, 1, 1, 7, 9)), models.mass_action_3(6)):
        b = np.asarray(m.bounds, np.int32)
        sv, sc, sr = m.stoich_csr()
        vals = np.empty_like(m.tables)
        offs = np.empty((m.nr, m.ns), np.int32)
        tab = np.ascontiguousarray(m.tables)
        R.ref_sdkron_fill(m.ns, b.ctypes.data, m.nr, sv.ctypes.data, sc.ctypes.data, sr.ctypes.data,
                          tab.ctypes.data, vals.ctypes.data, offs.ctypes.data)
        assert np.array_equal(vals, m.tables)
        assert np.array_equal(offs, -m.nu)


def test_toggle_tables_from_oracle_match_model():
    m = models.toggle((31, 31))
    assert np.array_equal(oracle.toggle_factor_tables([31, 31]), m.tables)


def test_csr_zero_vector_and_cross_format():
    """tests/test_fsp_mat.cu:153-201: A*0 = 0; the propensity-function CSR and the factor-table
    (Kronecker) form agree to 1e-14 in l2 at x = 1."""
    m = models.toggle((31, 31))
    c = m.coefs(1.0)
    A_fun = oracle.assemble_model(m, oracle.PROP_TOGGLE)
    A_tab = oracle.assemble_model(m, oracle.PROP_TABLES)
    n = m.n_states
    assert np.abs(A_fun.spmv(c, np.zeros(n))).sum() == 0.0
    y1 = A_fun.spmv(c, np.ones(n))
    y2 = A_tab.spmv(c, np.ones(n))
    assert np.linalg.norm(y1 - y2) <= 1e-14


def test_csr_structure():
    """Per-reaction CSR rows hold the diagonal -a_r(x) and a_r(x - nu_r) in column order
    (src/fspmat_csr_kernels.cu:53-94); column sums are <= 0 (probability leaks at the boundary)."""
    m = models.birth_death_2()
    A = oracle.assemble_model(m)
    for r in range(m.nr):
        rp = A.rowptr[r]
        assert rp[0] == 0 and np.all(np.diff(rp) >= 1) and np.all(np.diff(rp) <= 2)
        rows, cols, vals = A.entries(r)
        assert np.all(np.diff(rows * (m.n_states + 1) + cols) > 0)  # sorted, unique per row
        d = rows == cols
        assert np.all(vals[d] <= 0) and np.all(vals[~d] >= 0)
    S = A.to_scipy(m.coefs(0))
    assert np.asarray(S.sum(axis=0)).max() <= 1e-12


def test_oracle_expm_matches_scipy():
    import scipy.linalg as sla
    rng = np.random.default_rng(0)
    for k, s in [(4, 0.1), (32, 3.0), (32, 50.0)]:
        A = rng.standard_normal((k, k)) * s
        E = sla.expm(A)
        assert np.abs(oracle.expm(A) - E).max() <= 1e-12 * np.abs(E).max()


def test_oracle_expv_matches_scipy_expm_multiply():
    import scipy.sparse.linalg as spla
    m = models.birth_death_2()
    A = oracle.assemble_model(m)
    c = m.coefs(0)
    w, st, rc = oracle.expv(A, c, 10.0, m.p0(), m=30, tol=1e-8)
    assert rc == 0 and st["t_now"] == 10.0
    ws = spla.expm_multiply(A.to_scipy(c) * 10.0, m.p0())
    assert np.abs(w - ws).sum() <= 1e-8


@pytest.mark.parametrize("m_dim,q", [(30, 2), (60, 3), (60, 4)])
def test_oracle_iop_expv_matches_scipy_on_stiff_network(m_dim, q):
    """Incomplete orthogonalisation (src/KryExpvFSP.cu:74, q vectors) as the 255^3 expmv leg runs it
    (m = 60, q = 3) and as the reference's own test does (m = 30, q = 2), on a 21^3 box of the same
    stiff 3-species network to t = 0.2: within the Krylov tolerance of SciPy's expm_multiply."""
    import scipy.sparse.linalg as spla
    m = models.mass_action_3(bounds=(20, 20, 20))
    A = oracle.assemble_model(m)
    c = m.coefs(0)
    w, st, rc = oracle.expv(A, c, 0.2, m.p0(), m=m_dim, tol=1e-8, iop=True, q_iop=q)
    assert rc == 0 and st["t_now"] == 0.2
    ws = spla.expm_multiply(A.to_scipy(c) * 0.2, m.p0())
    assert np.abs(w - ws).sum() <= 1e-8


def test_oracle_mass_conservation_reference_case():
    """tests/test_kry_expv.cu:80-110: toggle on 257^2 states, t = 8 h, m = 30, tol 1e-8, IOP q = 2;
    |1 - sum v| <= 1e-10."""
    m = models.toggle((256, 256))
    A = oracle.assemble_model(m)
    w, st, rc = oracle.expv(A, m.coefs(0), 8 * 3600.0, m.p0(), m=30, tol=1e-8, iop=True, q_iop=2)
    assert rc == 0
    assert abs(1.0 - w.sum()) <= 1e-10


def test_oracle_step_limit_and_zero_vector():
    m = models.birth_death_2()
    A = oracle.assemble_model(m)
    _, _, rc = oracle.expv(A, m.coefs(0), 10.0, m.p0(), m=30, tol=1e-8, max_nstep=2)
    assert oracle.ORC_ERR[rc] == "STEP_LIMIT"
    w, st, rc = oracle.expv(A, m.coefs(0), 10.0, np.zeros(m.n_states))
    assert rc == 0 and not w.any()


def test_oracle_bdf_change_matrix_properties():
    """Step-change matrix of the backward-difference BDF: identity at rho = 1 and a group in rho
    (changing by a then by b equals changing by a*b)."""
    for k in range(1, 6):
        assert np.abs(oracle.bdf_change_matrix(k, 1.0) - np.eye(k + 1)).max() <= 1e-12
        Ta, Tb, Tab = (oracle.bdf_change_matrix(k, r) for r in (0.5, 1.7, 0.85))
        assert np.abs(Tb @ Ta - Tab).max() <= 1e-12 * max(1.0, np.abs(Tab).max())


def test_oracle_bdf_matches_krylov_time_invariant():
    m = models.birth_death_2()
    A = oracle.assemble_model(m)
    Y, st, rc = oracle.bdf(A, m.coefs(0), 0.0, m.p0(), [1.0, 10.0], rtol=1e-8, atol=1e-14)
    assert rc == 0 and st["t"] == 10.0 and st["order"] >= 3
    for t, y in zip((1.0, 10.0), Y):
        ref, _, rc = oracle.expv(A, m.coefs(0), t, m.p0(), tol=1e-13)
        assert np.abs(y - ref).sum() <= 1e-7


def test_oracle_bdf_matches_scipy_time_varying():
    """The reference's CVODE case (tests/test_sundials.cu:55-64: toggle switch with c_r(t)) on a
    32^2 box, against SciPy's Radau at rtol 1e-12."""
    import scipy.integrate as si
    m = models.toggle((31, 31), time_varying=True)
    A = oracle.assemble_model(m)
    times = [50.0, 500.0]
    Y, st, rc = oracle.bdf(A, m.coefs, 0.0, m.p0(), times, rtol=1e-9, atol=1e-14)
    assert rc == 0 and st["n_lin_fail"] == 0
    Ms = [A.to_scipy(np.eye(A.nr)[r]) for r in range(A.nr)]

    def jac(t, y):
        c = m.coefs(t)
        return sum(c[r] * Ms[r] for r in range(A.nr))
    sol = si.solve_ivp(lambda t, y: jac(t, y) @ y, (0.0, times[-1]), m.p0(), method="Radau", t_eval=times,
                       rtol=1e-12, atol=1e-16, jac=jac)
    assert sol.status == 0
    for k in range(len(times)):
        assert np.abs(Y[k] - sol.y[:, k]).sum() <= 1e-7


def test_oracle_bdf_limits():
    m = models.birth_death_2()
    A = oracle.assemble_model(m)
    _, _, rc = oracle.bdf(A, m.coefs(0), 0.0, m.p0(), [10.0], max_steps=3)
    assert oracle.ORC_ERR[rc] == "STEP_LIMIT"
    Y, st, rc = oracle.bdf(A, m.coefs(0), 0.0, m.p0(), [0.0, 0.0])
    assert rc == 0 and st["n_steps"] == 0 and np.array_equal(Y[1], m.p0())


def test_oracle_gradients_match_central_differences():
    """The oracle's two gradient routines, the checkers of the device adjoint: forward sensitivities
    by expm_multiply and by this oracle's Krylov expv on the augmented system agree with each other
    and with central differences of the oracle's log-likelihood in log c_r (5-species gene network,
    512 states, counts marginalised over the 8 gene states at 3 times)."""
    from scipy.sparse.linalg import expm_multiply
    m = models.gene_expression((1, 1, 1, 7, 7), time_varying=False)
    csr = oracle.assemble_model(m)
    c = m.coefs(0)
    times = np.array([1.0, 4.0, 12.0])
    block = 8
    rng = np.random.default_rng(5)
    A = csr.to_scipy(c).tocsc()
    p, t_prev, counts = m.p0(), 0.0, []
    for t in times:  # multinomial histograms of the exact marginals
        p = expm_multiply((t - t_prev) * A, p)
        t_prev = t
        q = np.clip(p.reshape(-1, block).sum(axis=1), 0.0, None)
        counts.append(rng.multinomial(300, q / q.sum()).astype(float))
    counts = np.array(counts)
    ll, g = oracle.loglik_grad_forward(csr, c, times, m.p0(), counts, block)
    rates = [0, 5, 8, 11]
    ll_k, g_k = oracle.loglik_grad_forward_krylov(csr, c, times, m.p0(), counts, block, rates)
    assert abs(ll_k - ll) <= 1e-10 * abs(ll)
    h = 1e-5
    for r in rates:
        cp, cm = c.copy(), c.copy()
        cp[r] *= np.exp(h)
        cm[r] *= np.exp(-h)
        fd = (oracle.loglik(csr, cp, times, m.p0(), counts, block) -
              oracle.loglik(csr, cm, times, m.p0(), counts, block)) / (2 * h)
        assert abs(g[r] - fd) <= 1e-6 * max(1.0, abs(fd)), (r, g[r], fd)
        assert abs(g_k[r] - g[r]) <= 1e-9 * max(1.0, abs(g[r])), (r, g_k[r], g[r])

