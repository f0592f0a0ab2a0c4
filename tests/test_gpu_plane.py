"""The runtime-specialised plane kernel of KRONECKER generators against the oracle (gpu).

Near-neighbour networks of 2 or 3 species with an even species-0 extent are served by a kernel
compiled per network at create time (NVRTC); everything else by the general kernel.  These tests
check that the plane kernel is the one in use where it should be, and that it reproduces the
oracle's generator (fspmat_csr_kernels.cu:53-94 restated) to the matvec bar on box shapes that
exercise every edge of its tiling: partial x0 chunks, row counts the tile height does not divide,
a single plane, one pair of positions, and random stoichiometries (every in-plane and cross-plane
neighbour offset, shared offsets, grouped and ungrouped diagonals).
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


def random_network(bounds, nr, seed, shared_inner=True):
    """nr reactions with net changes in {-1, 0, 1} per species and positive factor tables; when
    shared_inner, some reactions reuse another's species-0 table (diagonal groups)."""
    rng = np.random.default_rng(seed)
    ns = len(bounds)
    nu = np.zeros((nr, ns), np.int32)
    for r in range(nr):
        while not nu[r].any():
            nu[r] = rng.integers(-1, 2, ns)
    stride = sum(b + 1 for b in bounds)
    tables = rng.uniform(0.2, 3.0, (nr, stride))
    if shared_inner:
        for r in range(1, nr):
            if rng.uniform() < 0.4:
                tables[r, :bounds[0] + 1] = tables[rng.integers(0, r), :bounds[0] + 1]
    rates = 10.0 ** rng.uniform(-1, 1, nr)
    return models.CMEModel(f"random{seed}", list(bounds), nu, tables, rates)


def check(m, accumulate_cases=True):
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    csr = oracle.assemble_model(m)
    rng = np.random.default_rng(11)
    x = rng.uniform(0, 1, m.n_states)
    y0 = rng.uniform(-1, 1, m.n_states)
    c = m.coefs(0.0)
    scale = csr.abs_spmv(c, x).max()
    y = dev(y0)
    A.apply(dev(x), y, coefs=c, beta=1.0)
    err = np.abs(host(y) - csr.spmv(c, x, y0, beta=1.0)).max() / scale
    assert err <= MATVEC_RTOL, (m.name, m.bounds, "accumulate", err)
    if accumulate_cases:
        y = dev(np.full(m.n_states, np.nan))  # the overwrite form must not read y
        A.apply(dev(x), y, coefs=c, alpha=-0.7, beta=0.0)
        err = np.abs(host(y) - csr.spmv(-0.7 * c, x)).max() / scale
        assert err <= MATVEC_RTOL, (m.name, m.bounds, "overwrite", err)
    assert A.watchdog() == 0  # no bounded barrier wait of the TMA ring expired
    return A


PLANE_SHAPES = [
    ("bd2", models.birth_death_2),
    ("toggle31", lambda: models.toggle((31, 31))),
    ("ma3_64", lambda: models.mass_action_3(63)),
    ("ma3_rows_odd", lambda: models.mass_action_3(bounds=(63, 40, 17))),   # 41 rows: tile height 1
    ("ma3_chunk_partial", lambda: models.mass_action_3(bounds=(95, 33, 9))),  # 96 = 64 + 32 positions
    ("ma3_one_plane", lambda: models.mass_action_3(bounds=(31, 31, 0))),
    ("ma3_one_pair", lambda: models.mass_action_3(bounds=(1, 5, 7))),
    ("ma3_tall", lambda: models.mass_action_3(bounds=(17, 3, 200))),
    ("ma3_wide", lambda: models.mass_action_3(bounds=(1023, 3, 5))),     # 16 warps per tile
]


@pytest.mark.parametrize("name,make", PLANE_SHAPES)
def test_plane_kernel_matches_oracle(cuda, name, make):
    A = check(make())
    assert "plane kernel" in A.describe() and "not used" not in A.describe(), A.describe()


@pytest.mark.parametrize("seed", range(8))
def test_plane_kernel_random_networks(cuda, seed):
    rng = np.random.default_rng(100 + seed)
    ns = 2 if seed % 4 == 0 else 3
    bounds = [int(2 * rng.integers(1, 40) - 1)] + [int(rng.integers(0, 30)) for _ in range(ns - 1)]
    nr = int(rng.integers(1, 17))
    A = check(random_network(bounds, nr, seed, shared_inner=seed % 2 == 0))
    assert "plane kernel" in A.describe(), A.describe()


def test_plane_kernel_many_reactions(cuda):
    """32 reactions: more row words per tile than a warp has lanes."""
    A = check(random_network((41, 9, 12), 32, 7))
    assert "plane kernel" in A.describe(), A.describe()


def test_general_kernel_where_the_plane_kernel_does_not_apply(cuda, monkeypatch):
    for m, why in ((models.mass_action_3(bounds=(20, 9, 9)), "odd"),
                   (models.gene_expression(), "species"),
                   (random_network((7, 7, 7), 3, 1), None)):
        if why is None:  # a change of 2 molecules
            m.nu[0, 1] = 2
        A = check(m)
        assert "not used" in A.describe(), A.describe()
    monkeypatch.setenv("CUFSP_PLANE", "0")
    A = check(models.mass_action_3(31))
    assert "not used" in A.describe()


def test_plane_and_general_kernels_agree(cuda, monkeypatch):
    m = models.mass_action_3(bounds=(127, 63, 31))
    csr = oracle.assemble_model(m)
    x = np.random.default_rng(3).uniform(0, 1, m.n_states)
    c = m.coefs(0.0)
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    ya = dev(np.zeros(m.n_states))
    A.apply(dev(x), ya, coefs=c, beta=0.0)
    monkeypatch.setenv("CUFSP_PLANE", "0")
    B = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    yb = dev(np.zeros(m.n_states))
    B.apply(dev(x), yb, coefs=c, beta=0.0)
    assert "plane kernel" in A.describe() and "not used" in B.describe()
    assert np.abs(host(ya) - host(yb)).max() <= 2 * MATVEC_RTOL * csr.abs_spmv(c, x).max()


def test_plane_kernel_host_pipeline_slabs(cuda):
    """cufsp_mat_action_host applies the plane kernel slab by slab (whole planes per slab)."""
    import torch
    m = models.mass_action_3(bounds=(63, 31, 40))
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    csr = oracle.assemble_model(m)
    rng = np.random.default_rng(5)
    x = rng.uniform(0, 1, m.n_states)
    y0 = rng.uniform(-1, 1, m.n_states)
    xh = torch.as_tensor(x).pin_memory()
    yh = torch.as_tensor(y0.copy()).pin_memory()
    A.action_host(0.0, xh, yh)
    c = m.coefs(0.0)
    err = np.abs(yh.numpy() - csr.spmv(c, x, y0, beta=1.0)).max() / csr.abs_spmv(c, x).max()
    assert err <= MATVEC_RTOL, err


def test_plane_kernel_is_deterministic(cuda):
    """Two applications give bit-identical results (no reduction order depends on scheduling)."""
    m = models.mass_action_3(bounds=(63, 63, 63))
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    x = dev(np.random.default_rng(9).uniform(0, 1, m.n_states))
    y1, y2 = dev(np.zeros(m.n_states)), dev(np.zeros(m.n_states))
    A.apply(x, y1, coefs=m.coefs(0.0), beta=0.0)
    A.apply(x, y2, coefs=m.coefs(0.0), beta=0.0)
    assert np.array_equal(host(y1), host(y2))


def check_general(m, x=None):
    """A KRONECKER generator not served by the plane kernel against the oracle (both forms)."""
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    csr = oracle.assemble_model(m)
    rng = np.random.default_rng(12)
    x = rng.uniform(0, 1, m.n_states) if x is None else x
    y0 = rng.uniform(-1, 1, m.n_states)
    c = m.coefs(0.0)
    scale = csr.abs_spmv(c, x).max()
    for beta in (0.0, 1.0):
        y = dev(y0)
        A.apply(dev(x), y, coefs=c, beta=beta)
        ref = csr.spmv(c, x, y0 if beta else None, beta=beta)
        err = np.abs(host(y) - ref).max()
        assert err <= MATVEC_RTOL * (scale + (np.abs(y0).max() if beta else 0.0)), (m.name, m.bounds, beta, err)
    return A


@pytest.mark.parametrize("case", ["gene", "odd_states", "big_change", "random5", "toggle_no_plane"])
def test_specialised_general_kernel_matches_oracle(cuda, case, monkeypatch):
    """The KRONECKER kernel specialised per network and box (factor kinds ones / identity / table as
    constants; opt-in for the forward action, CUFSP_KRON_RTC=1) on networks outside the plane kernel's
    shape: 5 species, an odd state count, a change of 2 molecules, random 4-species networks, and a
    plane-shaped network with the plane kernel off."""
    monkeypatch.setenv("CUFSP_KRON_RTC", "1")
    if case == "gene":
        m = models.gene_expression((1, 1, 1, 63, 40), time_varying=False)
    elif case == "odd_states":
        m = models.mass_action_3(bounds=(6, 8, 4))  # 7 * 9 * 5 = 315 states, a change of 2 molecules
        m.nu[0, 0] = 2
    elif case == "big_change":
        m = random_network((9, 7, 11), 5, 4)
        m.nu[1, 2] = -2
        m.nu[3, 0] = 3
    elif case == "random5":
        m = random_network((3, 4, 2, 5, 6), 7, 9)
    else:
        monkeypatch.setenv("CUFSP_PLANE", "0")
        m = models.toggle((63, 40))
    A = check_general(m)
    assert "specialised" in A.describe(), A.describe()


def test_generic_kernel_remains(cuda, monkeypatch):
    """By default (and with the specialised kernels switched off) the generic k_kron_mv serves the
    forward action of networks outside the plane kernel's shape, to the same bar."""
    monkeypatch.setenv("CUFSP_PLANE", "0")
    A = check_general(models.gene_expression((1, 1, 1, 20, 11), time_varying=False))
    assert "k_kron_mv" in A.describe(), A.describe()
    monkeypatch.setenv("CUFSP_KRON_RTC", "0")
    for m in (models.gene_expression((1, 1, 1, 40, 23), time_varying=False), models.mass_action_3(bounds=(20, 9, 9))):
        A = check_general(m)
        assert "k_kron_mv" in A.describe(), A.describe()
