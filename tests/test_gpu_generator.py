"""Generator action and state enumeration on the GPU, through the C ABI, against the oracle (gpu)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from conftest import require_ref
from cuda_fsp_b200 import FSPMat, MatrixFormat, get_states, models

pytestmark = pytest.mark.gpu

# Matvec parity bar: max_i |y_gpu - y_oracle|_i <= 1e-13 * max_i (sum_r |c_r| |A_r| |x|)_i
MATVEC_RTOL = 1e-13


def dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def check_matvec(A: FSPMat, csr, coefs, x, y0=None, accumulate=True, alpha=1.0):
    import torch
    y = dev(np.zeros(csr.n) if y0 is None else y0)
    if accumulate:
        A.apply(dev(x), y, coefs=coefs, alpha=alpha, beta=1.0)
    else:
        A.apply(dev(x), y, coefs=coefs, alpha=alpha, beta=0.0)
    got = host(y)
    ref = csr.spmv(np.asarray(coefs) * alpha, x, y0 if (accumulate and y0 is not None) else None,
                   beta=1.0 if (accumulate and y0 is not None) else 0.0)
    scale = max(csr.abs_spmv(np.asarray(coefs) * alpha, x).max(), 1e-300)
    err = np.abs(got - ref).max() / scale
    assert err <= MATVEC_RTOL, err
    return got


def prop_bound(m, coefs):
    """sum_r |c_r| prod_s max_x |f_{r,s}(x)|: an upper bound of the total propensity on the box."""
    tot = 0.0
    for r in range(m.nr):
        p, off = abs(coefs[r]), 0
        for b in m.bounds:
            p *= np.abs(m.tables[r, off:off + b + 1]).max()
            off += b + 1
        tot += p
    return tot


SMALL_MODELS = [
    ("toggle31", lambda: models.toggle((31, 31))),
    ("toggle_odd", lambda: models.toggle((40, 22))),
    ("bd2", models.birth_death_2),
    ("gene", models.gene_expression),
    ("gene_odd", lambda: models.gene_expression((1, 1, 1, 66, 93))),
    ("ma3_small", lambda: models.mass_action_3(20)),
    ("ma3_odd", lambda: models.mass_action_3(bounds=(20, 17, 13))),
]


@pytest.mark.parametrize("name,make", SMALL_MODELS)
@pytest.mark.parametrize("fmt", [MatrixFormat.KRONECKER, MatrixFormat.HYB])
def test_matvec_matches_oracle(cuda, name, make, fmt):
    m = make()
    A = FSPMat.from_model(m, fmt)
    csr = oracle.assemble_model(m)
    rng = np.random.default_rng(7)
    x = rng.uniform(0, 1, m.n_states)
    c = m.coefs(6.0)
    y0 = rng.uniform(-1, 1, m.n_states)
    check_matvec(A, csr, c, x, y0=y0, accumulate=True)
    check_matvec(A, csr, c, x, accumulate=False, alpha=0.37)
    # x = 1 (column-sum check of the reference tests) and x = 0
    check_matvec(A, csr, c, np.ones(m.n_states), accumulate=False)
    z = dev(y0)
    A.apply(dev(np.zeros(m.n_states)), z, coefs=c, beta=1.0)
    assert np.array_equal(host(z), y0)


MARCH_MODELS = [
    ("toggle31", lambda: models.toggle((31, 31))),
    ("bd2", models.birth_death_2),
    ("ma3_32", lambda: models.mass_action_3(31)),
    ("ma3_uneven", lambda: models.mass_action_3(bounds=(63, 40, 17))),  # 41 rows/plane: partial tile
]


@pytest.mark.parametrize("name,make", MARCH_MODELS)
def test_tma_march_path_matches_oracle_and_fallback(cuda, name, make, monkeypatch):
    """The TMA-fed marching kernel and the register/L1 kernel give the oracle's result; the
    marching kernel's bounded barrier waits never expire."""
    m = make()
    csr = oracle.assemble_model(m)
    rng = np.random.default_rng(13)
    x = rng.uniform(0, 1, m.n_states)
    y0 = rng.uniform(-1, 1, m.n_states)
    c = m.coefs(0)
    monkeypatch.setenv("CUFSP_KRON_MARCH", "1")
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    got_march = check_matvec(A, csr, c, x, y0=y0, accumulate=True)
    check_matvec(A, csr, c, x, accumulate=False, alpha=-2.5)
    assert A.watchdog() == 0
    monkeypatch.setenv("CUFSP_KRON_MARCH", "0")
    B = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    got_ldg = check_matvec(B, csr, c, x, y0=y0, accumulate=True)
    scale = csr.abs_spmv(c, x).max()
    assert np.abs(got_march - got_ldg).max() <= 2 * MATVEC_RTOL * scale


def test_vectors_only_8_byte_aligned(cuda):
    """x and y that start 8 bytes past a 16-byte boundary (e.g. Krylov basis vectors of odd length)
    are handled: the paired-load and TMA paths step aside for the scalar kernel."""
    import torch
    for m in (models.birth_death_2(), models.mass_action_3(31)):
        A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
        csr = oracle.assemble_model(m)
        n = m.n_states
        rng = np.random.default_rng(17)
        x = rng.uniform(0, 1, n)
        bx = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
        by = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
        bx[1:] = torch.as_tensor(x, device="cuda")
        A.apply(bx[1:], by[1:], coefs=m.coefs(0), beta=0.0)
        ref = csr.spmv(m.coefs(0), x)
        assert np.abs(host(by[1:]) - ref).max() <= MATVEC_RTOL * csr.abs_spmv(m.coefs(0), x).max()
        assert host(by)[0] == 0.0


def test_action_uses_time_coefficients(cuda):
    """FSPMat::action(t, x, y): y += A(t) x with c(t) from the TcoefFun (src/FSPMat.cu:102-105)."""
    m = models.gene_expression()
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    csr = oracle.assemble_model(m)
    x = np.random.default_rng(2).uniform(0, 1, m.n_states)
    for t in (0.0, 5.0, 30.0):
        y = dev(np.zeros(m.n_states))
        A.action(t, dev(x), y)
        ref = csr.spmv(m.coefs(t), x)
        assert np.abs(host(y) - ref).max() <= MATVEC_RTOL * csr.abs_spmv(m.coefs(t), x).max()


def test_sparse_propensity_table_is_bit_exact(cuda):
    """The sparse format's stored a_r(x_i) equal the oracle CSR diagonal entries bit for bit."""
    for m in (models.gene_expression((1, 1, 1, 30, 20)), models.mass_action_3(12), models.toggle((31, 31))):
        A = FSPMat.from_model(m, MatrixFormat.HYB)
        P = host(A.export_propensities())
        csr = oracle.assemble_model(m)
        for r in range(m.nr):
            rows, cols, vals = csr.entries(r)
            d = rows == cols
            assert np.array_equal(-vals[d], P[r])


def test_device_propfun_path(cuda, testmodels):
    """PropFun (a __device__ function address) drives the sparse build, as in the reference's HYB
    path (src/fspmat_hyb_kernels.cu:44-53); checked against the oracle's C propensities."""
    for kind, getter in ((oracle.PROP_TOGGLE, testmodels.tm_toggle_propfn), (oracle.PROP_NONFACT, testmodels.tm_nonfact_propfn)):
        m = models.toggle((31, 45))
        fn = getter()
        assert fn
        A = FSPMat(m.nr, m.ns, m.bounds, m.stoich_csr(), m.coefs, fn, MatrixFormat.HYB, lib=testmodels)
        csr = oracle.assemble_model(m, kind)
        P = host(A.export_propensities())
        for r in range(m.nr):
            rows, cols, vals = csr.entries(r)
            d = rows == cols
            np.testing.assert_allclose(-vals[d], P[r], rtol=4e-16, atol=0)
        x = np.random.default_rng(5).uniform(0, 1, m.n_states)
        check_matvec(A, csr, m.coefs(0), x, accumulate=False)


def test_kron_equals_hyb_reference_tolerances(cuda):
    """tests/test_fsp_mat.cu:188-201: HYB and KRON agree to 1e-12 in l2 at x = 1; A 0 = 0."""
    m = models.toggle((31, 31))
    K = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    H = FSPMat.from_model(m, MatrixFormat.HYB)
    n = m.n_states
    w = [dev(np.zeros(n)) for _ in range(2)]
    K.action(1.0, dev(np.zeros(n)), w[0])
    H.action(1.0, dev(np.zeros(n)), w[1])
    assert abs(host(w[0]).sum()) <= 1e-14 and abs(host(w[1]).sum()) <= 1e-14
    K.action(1.0, dev(np.ones(n)), w[0])
    H.action(1.0, dev(np.ones(n)), w[1])
    assert np.linalg.norm(host(w[0]) - host(w[1])) <= 1e-12


def test_against_reference_gpu_kernels(cuda):
    """The reference's own HYB and Kronecker kernels (built from its sources into oracle/_ref) on
    sizes they handle (multiples of 1024 states)."""
    R = require_ref()
    rng = np.random.default_rng(11)
    # HYB with the toggle PropFun, 32x32 = 1024 states
    m = models.toggle((31, 31))
    b = np.asarray(m.bounds, np.int32)
    x = rng.uniform(0, 1, m.n_states)
    c = np.ascontiguousarray(m.coefs(0))
    y_ref = np.zeros(m.n_states)
    assert R.ref_gpu_hyb_toggle(b.ctypes.data, c.ctypes.data, x.ctypes.data, y_ref.ctypes.data) == 0
    for fmt in (MatrixFormat.KRONECKER, MatrixFormat.HYB):
        A = FSPMat.from_model(m, fmt)
        y = dev(np.zeros(m.n_states))
        A.action(0.0, dev(x), y)
        scale = oracle.assemble_model(m).abs_spmv(c, x).max()
        assert np.abs(host(y) - y_ref).max() <= 1e-13 * scale
    # HYB built by the reference's own fill kernel from a factor-table PropFun, on the 3-species 32^3
    # and the 5-species gene workloads
    for m in (models.mass_action_3(31), models.gene_expression((1, 1, 1, 31, 31), time_varying=False)):
        b = np.asarray(m.bounds, np.int32)
        sv, sc, sr = m.stoich_csr()
        tab = np.ascontiguousarray(m.tables)
        c = np.ascontiguousarray(m.coefs(0))
        x = rng.uniform(0, 1, m.n_states)
        y_ref = np.zeros(m.n_states)
        assert R.ref_gpu_hyb_tables(m.ns, m.nr, b.ctypes.data, sv.ctypes.data, sc.ctypes.data, sr.ctypes.data,
                                    tab.ctypes.data, c.ctypes.data, x.ctypes.data, y_ref.ctypes.data, 0, None) == 0
        scale = oracle.assemble_model(m).abs_spmv(c, x).max()
        for fmt in (MatrixFormat.KRONECKER, MatrixFormat.HYB):
            A = FSPMat.from_model(m, fmt)
            y = dev(np.zeros(m.n_states))
            A.action(0.0, dev(x), y)
            assert np.abs(host(y) - y_ref).max() <= 1e-13 * scale, (m.name, fmt)
    # Kronecker on the 2-species (32,768 states) and 3-species 32^3 workloads
    for m in (models.birth_death_2(), models.mass_action_3(31)):
        b = np.asarray(m.bounds, np.int32)
        sv, sc, sr = m.stoich_csr()
        tab = np.ascontiguousarray(m.tables)
        c = np.ascontiguousarray(m.coefs(0))
        x = rng.uniform(0, 1, m.n_states)
        y_ref = np.zeros(m.n_states)
        assert R.ref_gpu_kron(m.ns, m.nr, b.ctypes.data, sv.ctypes.data, sc.ctypes.data, sr.ctypes.data, tab.ctypes.data,
                              c.ctypes.data, x.ctypes.data, y_ref.ctypes.data) == 0
        A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
        y = dev(np.zeros(m.n_states))
        A.action(0.0, dev(x), y)
        scale = oracle.assemble_model(m).abs_spmv(c, x).max()
        assert np.abs(host(y) - y_ref).max() <= 1e-13 * scale


def test_full_size_properties(cuda):
    """16,777,216 states (255^3): linearity, column sums and determinism, and agreement with the
    reference Kronecker kernel on a random vector."""
    import torch
    m = models.mass_action_3()
    n = m.n_states
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    g = torch.Generator(device="cuda").manual_seed(3)
    x1 = torch.rand(n, dtype=torch.float64, device="cuda", generator=g)
    x2 = torch.rand(n, dtype=torch.float64, device="cuda", generator=g)
    y1, y2, y3 = (torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(3))
    c = m.coefs(0)
    A.apply(x1, y1, coefs=c)
    A.apply(x2, y2, coefs=c)
    A.apply(2.0 * x1 - 3.0 * x2, y3, coefs=c)
    bound = prop_bound(m, c)  # >= max_i sum_r |c_r| (|A_r| |x|)_i / 2 for x in [0, 1]
    assert (y3 - (2.0 * y1 - 3.0 * y2)).abs().max().item() <= 1e-13 * 2 * bound * 5
    y1b = torch.zeros_like(y1)
    A.apply(x1, y1b, coefs=c)
    assert torch.equal(y1, y1b)  # deterministic, no atomics
    # mass balance: 1^T A p = -(outflow through the box boundary) <= 0
    p = torch.as_tensor(m.p0(), device="cuda")
    yp = torch.zeros_like(p)
    A.apply(p, yp, coefs=c)
    assert yp.sum().item() <= 1e-12
    R = require_ref()
    b = np.asarray(m.bounds, np.int32)
    sv, sc, sr = m.stoich_csr()
    tab = np.ascontiguousarray(m.tables)
    cc = np.ascontiguousarray(c)
    xh = x1.cpu().numpy()
    y_ref = np.zeros(n)
    assert R.ref_gpu_kron(m.ns, m.nr, b.ctypes.data, sv.ctypes.data, sc.ctypes.data, sr.ctypes.data, tab.ctypes.data,
                          cc.ctypes.data, xh.ctypes.data, y_ref.ctypes.data) == 0
    assert np.abs(host(y1) - y_ref).max() <= MATVEC_RTOL * 2 * bound


def test_action_host_buffers(cuda):
    """cufsp_mat_action_host: pinned host x, y; pipelined H2D/compute/D2H equals the device path."""
    import torch
    for m in (models.gene_expression(), models.mass_action_3(63)):
        for fmt in (MatrixFormat.KRONECKER, MatrixFormat.HYB):
            A = FSPMat.from_model(m, fmt)
            rng = np.random.default_rng(4)
            x = torch.from_numpy(rng.uniform(0, 1, m.n_states)).pin_memory()
            y = torch.from_numpy(rng.uniform(-1, 1, m.n_states)).pin_memory()
            yd = y.cuda()
            A.action(2.0, x.cuda(), yd)
            A.action_host(2.0, x, y)
            # the slab pipeline and the whole-vector launch may use different kernels (summation order)
            scale = oracle.assemble_model(m).abs_spmv(m.coefs(2.0), x.numpy()).max()
            assert (y - yd.cpu()).abs().max().item() <= MATVEC_RTOL * scale


def test_enumeration_known_answer_on_gpu(cuda):
    """tests/test_fsp_get_states.cu: (1023, 1023, 3) bit-exact, plus uneven boxes; and the reference
    fsp_get_states kernel itself where the shim is built."""
    for b in ([1023, 1023, 3], [6, 0, 9, 2], [100000], [1, 1, 1, 127, 127]):
        got = get_states(b).cpu().numpy()
        assert np.array_equal(got, oracle.get_states(b))
    R = require_ref()
    b = np.asarray([1023, 1023, 3], np.int32)
    out = np.empty((1024 * 1024 * 4, 3), np.int32)
    assert R.ref_gpu_get_states(3, b.ctypes.data, out.ctypes.data) == 0
    assert np.array_equal(out, oracle.get_states(b))
