"""The row kernels of KRONECKER generators (cufsp_kron_rows_*, compiled per network and box) against
the oracle (gpu).

The forward action y = alpha A x (+ y) of networks outside the plane kernel's shape, and the
transposed action y = alpha A^T x of every KRONECKER network, are served by kernels that fix the
inner species' factor products per lane and sweep the rows of the outer species.  These tests hold
them to the matvec bar of the oracle's generator (fspmat_csr_kernels.cu:53-94 restated) on boxes
that exercise partial row chunks, one and many inner species, 1 to 5 species, changes of more than
one molecule, both lane layouts and the default selection above 65,536 states.
"""
import numpy as np
import pytest

import oracle
from cuda_fsp_b200 import FSPMat, MatrixFormat, models

pytestmark = pytest.mark.gpu

MATVEC_RTOL = 1e-13


def dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def random_network(bounds, nr, seed):
    """nr reactions with net changes in {-1, 0, 1} per species and positive factor tables, some of
    them the identity or all ones (the kernel folds those at compile time)."""
    rng = np.random.default_rng(seed)
    ns = len(bounds)
    nu = np.zeros((nr, ns), np.int32)
    for r in range(nr):
        while not nu[r].any():
            nu[r] = rng.integers(-1, 2, ns)
    offs = np.concatenate([[0], np.cumsum([b + 1 for b in bounds])])
    tables = rng.uniform(0.2, 3.0, (nr, int(offs[-1])))
    for r in range(nr):
        for s in range(ns):
            u = rng.uniform()
            if u < 0.3:
                tables[r, offs[s]:offs[s + 1]] = 1.0
            elif u < 0.5:
                tables[r, offs[s]:offs[s + 1]] = np.arange(bounds[s] + 1)
    rates = 10.0 ** rng.uniform(-1, 1, nr)
    return models.CMEModel(f"random{seed}", list(bounds), nu, tables, rates)


def one_species():
    """Birth-death on one species: a single row of inner positions."""
    nu = np.array([[1], [-1]], np.int32)
    tables = np.stack([np.ones(700), np.arange(700.0)])
    return models.CMEModel("birth_death_1", [699], nu, tables, np.array([4.0, 0.3]))


def check_rows(m, expect_rows=True):
    """Forward (both forms) and transposed action of m against the oracle; returns the generator."""
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    csr = oracle.assemble_model(m)
    rng = np.random.default_rng(21)
    x = rng.uniform(0, 1, m.n_states)
    y0 = rng.uniform(-1, 1, m.n_states)
    c = m.coefs(0.0)
    alpha = 0.75
    scale = csr.abs_spmv(c, x).max()
    for beta in (0.0, 1.0):
        y = dev(y0)
        A.apply(dev(x), y, coefs=c, alpha=alpha, beta=beta)
        ref = alpha * csr.spmv(c, x) + (y0 if beta else 0.0)
        err = np.abs(host(y) - ref).max()
        assert err <= MATVEC_RTOL * (scale + (np.abs(y0).max() if beta else 0.0)), (m.name, m.bounds, beta, err)
    S = csr.to_scipy(c)
    yt = dev(y0)
    A.apply_transpose(dev(x), yt, coefs=c, alpha=alpha)
    ref_t = alpha * (S.T @ x)
    scale_t = (abs(S).T @ x).max()
    err_t = np.abs(host(yt) - ref_t).max()
    assert err_t <= MATVEC_RTOL * scale_t, (m.name, m.bounds, "transpose", err_t)
    if expect_rows:
        assert "row kernel" in A.describe() or "plane kernel" in A.describe(), A.describe()
    return A


@pytest.mark.parametrize("vp", ["1", "2", "4"])
@pytest.mark.parametrize("case", ["gene", "odd_states", "big_change", "random4", "random5", "toggle_no_plane",
                                  "one_species"])
def test_row_kernels_match_oracle(cuda, case, vp, monkeypatch):
    monkeypatch.setenv("CUFSP_KRON_ROWS", "1")
    monkeypatch.setenv("CUFSP_KRON_ROWS_V", vp)
    if case == "gene":
        m = models.gene_expression((1, 1, 1, 63, 40), time_varying=False)
    elif case == "odd_states":
        m = models.mass_action_3(bounds=(6, 8, 4))  # 7 * 9 * 5 = 315 states, a change of 2 molecules
        m.nu[0, 0] = 2
        monkeypatch.setenv("CUFSP_PLANE", "0")
    elif case == "big_change":
        m = random_network((9, 7, 11), 5, 4)
        m.nu[1, 2] = -2
        m.nu[3, 0] = 3
    elif case == "random4":
        m = random_network((5, 3, 6, 9), 11, 7)
    elif case == "random5":
        m = random_network((3, 4, 2, 5, 6), 7, 9)
    elif case == "toggle_no_plane":
        monkeypatch.setenv("CUFSP_PLANE", "0")
        m = models.toggle((63, 40))
    else:
        m = one_species()
    A = check_rows(m)
    if case not in ("one_species",) and "row kernel" not in A.describe():
        pytest.fail(A.describe())


def test_row_kernels_by_default_on_large_boxes(cuda, monkeypatch):
    """Above 65,536 states the row kernel is the default forward kernel of networks outside the plane
    kernel's shape (here the 5-species gene network, 131,072 states) and the transposed kernel of every
    network (a 41^3 box of the 3-species network, forward through the plane kernel)."""
    monkeypatch.delenv("CUFSP_KRON_ROWS", raising=False)
    A = check_rows(models.gene_expression((1, 1, 1, 127, 127), time_varying=False))
    assert "row kernel" in A.describe(), A.describe()
    A = check_rows(models.mass_action_3(bounds=(40, 40, 40)))
    assert "plane kernel" in A.describe(), A.describe()


def test_row_kernels_off(cuda, monkeypatch):
    """CUFSP_KRON_ROWS=0 returns the forward action to the generic kernel, to the same bar."""
    monkeypatch.setenv("CUFSP_KRON_ROWS", "0")
    A = check_rows(models.gene_expression((1, 1, 1, 127, 127), time_varying=False), expect_rows=False)
    assert "k_kron_mv" in A.describe(), A.describe()


def slab_case(case):
    if case == "gene":  # rows of 8 x 16 = 128 positions, 1,200 rows
        return models.gene_expression((1, 1, 1, 15, 1199), time_varying=False)
    if case == "random4":  # rows of 64 positions
        return random_network((3, 3, 3, 1299), 9, 17)
    if case == "random5":  # rows of 72 positions
        return random_network((2, 3, 1, 2, 1300), 7, 19)
    if case == "binary":  # three binary switches lead (sources by warp shuffle where one flips alone)
        m = random_network((1, 1, 1, 7, 1300), 10, 29)
        m.nu[1] = (0, 0, -1, 0, 0)
        m.nu[3] = (0, 1, 0, 0, 0)
        m.nu[7] = (1, 0, 0, 0, 0)
        m.nu[9] = (-1, 0, 0, 0, 0)
        m.nu[2] = (1, -1, 0, 0, 0)  # the same flat shift as reaction 9, another source pattern
        m.tables[2, 2:] = 1.0       # outer factors (and species 1) all ones: may share reaction 9's term
        m.tables[9, 2:] = 1.0
        return m
    m = random_network((15, 3, 1400), 6, 23)  # a change of 2 rows and one of 3 positions
    m.nu[1] = (0, 0, -2)
    m.nu[3] = (3, 0, 0)
    return m


@pytest.mark.parametrize("case", ["gene", "random4", "random5", "binary", "big_change"])
def test_slab_kernels_match_oracle(cuda, case, monkeypatch):
    """The slab kernels (rows streamed through shared memory by TMA bulk copies) on networks with
    at least 8 rows per CTA of a full grid: forward in both forms and transposed, to the matvec bar."""
    monkeypatch.delenv("CUFSP_KRON_ROWS", raising=False)
    A = check_rows(slab_case(case))
    assert "slab kernel" in A.describe(), A.describe()
    assert A.watchdog() == 0


def test_slab_falls_back_for_8_byte_aligned_vectors(cuda):
    """Vectors only 8-byte aligned (a Krylov basis vector at an odd offset) take the row kernel."""
    import torch
    m = slab_case("gene")
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    assert "slab kernel" in A.describe(), A.describe()
    csr = oracle.assemble_model(m)
    rng = np.random.default_rng(5)
    x = rng.uniform(0, 1, m.n_states)
    c = m.coefs(0.0)
    xb = torch.zeros(m.n_states + 1, dtype=torch.float64, device="cuda")
    yb = torch.zeros(m.n_states + 1, dtype=torch.float64, device="cuda")
    xb[1:] = dev(x)
    A.apply(xb[1:], yb[1:], coefs=c)
    err = np.abs(host(yb[1:]) - csr.spmv(c, x)).max()
    assert err <= MATVEC_RTOL * csr.abs_spmv(c, x).max(), err


def test_slab_watchdog(cuda, monkeypatch):
    """CUFSP_KRON_SLAB_WAIT_TRIES=0 at creation compiles the slab kernels with zero tries for the
    waits before each row, so every such wait gives up at once: the kernel drains its copies (with its
    normal bound), sets the watchdog word and returns; the context stays usable."""
    m = slab_case("gene")
    monkeypatch.setenv("CUFSP_KRON_SLAB_WAIT_TRIES", "0")
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    monkeypatch.delenv("CUFSP_KRON_SLAB_WAIT_TRIES")
    assert "slab kernel" in A.describe(), A.describe()
    y = dev(np.zeros(m.n_states))
    A.apply(dev(np.ones(m.n_states)), y, coefs=m.coefs(0.0))
    assert A.watchdog() == 1
    assert A.watchdog() == 0
    check_rows(m)  # a normal generator of the same network


@pytest.mark.parametrize("case", ["gene_rows_of_4096", "three_species_change_of_2", "three_species_plane"])
def test_tiled_slab_kernels_match_oracle(cuda, case, monkeypatch):
    """Rows longer than a CTA's tile (1024 positions): the slab kernels split every row into tiles,
    each staged with guards of up to 512 positions for its inner neighbours.  A 2.1M-state gene box
    (rows of 4096 positions, forward and transposed through tiles), a 3-species network with a change
    of 2 molecules (rows of 16,384 positions, neighbours 256 positions away), and the plane-shaped
    3-species network, whose transposed action goes through the tiled slab kernel."""
    monkeypatch.delenv("CUFSP_KRON_ROWS", raising=False)
    if case == "gene_rows_of_4096":
        m = models.gene_expression((1, 1, 1, 511, 511), time_varying=False)
    elif case == "three_species_change_of_2":
        m = models.mass_action_3(bounds=(127, 127, 127))
        m.nu[0] = (2, 0, 0)
        m.nu[6] = (0, -2, 1)
    else:
        m = models.mass_action_3(bounds=(127, 127, 127))
    A = check_rows(m)
    if case == "three_species_plane":
        assert "plane kernel" in A.describe(), A.describe()
    else:
        assert "slab kernel" in A.describe(), A.describe()
    assert A.watchdog() == 0
