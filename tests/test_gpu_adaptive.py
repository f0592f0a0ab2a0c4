"""FSP with an adaptively grown box (cufsp_adaptive_*) against the oracle on the largest box (gpu)."""
import numpy as np
import pytest

import oracle
from cuda_fsp_b200 import AdaptiveFSP, models

pytestmark = pytest.mark.gpu


def restrict(p_big, big_bounds, small_bounds):
    """The entries of a distribution on big_bounds that lie in small_bounds (species 0 fastest)."""
    shape_big = [b + 1 for b in reversed(big_bounds)]
    sl = tuple(slice(0, b + 1) for b in reversed(small_bounds))
    return p_big.reshape(shape_big)[sl].reshape(-1)


@pytest.mark.parametrize("case", ["bd2", "toggle"])
def test_adaptive_box_meets_fsp_tol(cuda, case):
    if case == "bd2":
        small, big, times, tol = models.birth_death_2(), (127, 255), [1.0, 4.0, 10.0], 1e-6
        small = models.mass_action((8, 8), small.nu, [[0, 0], [1, 0], [1, 0], [0, 1]], small.rates,
                                   name="birth_death_2")
    else:
        small, big, times, tol = models.toggle((4, 4)), (120, 120), [500.0, 2000.0, 8000.0], 1e-5
    S = AdaptiveFSP(small, big, times, fsp_tol=tol, grow=1.5)
    for i, t in enumerate(times):
        st = S.next_time()
        assert st["fsp_error"] <= tol * t / times[-1] + 1e-14 and not st["fsp_tol_exceeded"]
    p, bounds = S.solution()
    assert st["expansions"] >= 1 and all(b <= B for b, B in zip(bounds, big))
    # reference: the oracle on the largest box, restricted to the final box
    mbig = (models.toggle(big) if case == "toggle" else
            models.mass_action(big, small.nu, [[0, 0], [1, 0], [1, 0], [0, 1]], small.rates))
    csr = oracle.assemble_model(mbig)
    ref, _, rc = oracle.expv(csr, mbig.coefs(0), times[-1], mbig.p0(), m=30, tol=1e-10)
    assert rc == 0
    ref_box = restrict(ref, list(big), bounds)
    diff = np.abs(p.cpu().numpy() - ref_box).sum()
    # the truncated solution misses at most the probability that left its box (plus Krylov error)
    assert diff <= tol + 1e-7, diff


def test_adaptive_reports_when_the_box_cannot_grow(cuda):
    m = models.mass_action((6, 6), [[1, 0], [-1, 0], [0, 1], [0, -1]], [[0, 0], [1, 0], [1, 0], [0, 1]],
                           [10.0, 1.0, 0.5, 0.2])
    S = AdaptiveFSP(m, (9, 9), [5.0], fsp_tol=1e-8)
    st = S.next_time()
    assert st["fsp_tol_exceeded"] and st["bounds"][:2] == [9, 9]
