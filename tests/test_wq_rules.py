"""1-D weighted-quadrature rules: oracle pinned to the reference's own Python
twin (golden vectors), the defining exactness property, and the library's
host-side rule (yeti_wq_rule_1d, no GPU needed) against the oracle."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import wq_rules

CASES = [(2, 2), (2, 3), (2, 5), (2, 8), (3, 2), (3, 4), (3, 6), (3, 9),
         (4, 3), (4, 7), (4, 10)]
KEYS = ("B0", "B1", "W00", "W01", "W10", "W11")
# The local systems are solved by least squares / minimum norm; different
# solvers (LAPACK in the reference, lstsq / Householder QR here) agree to a
# few 1e-12 relative for p <= 4.
RULE_TOL = 1e-10


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLDEN, "wq_rules.npz"))


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("p,nel", CASES)
def test_oracle_rule_matches_reference_python_twin(golden, p, nel):
    """Golden vectors from base_functions.wq_find_basis_weights_opt
    (iga_wq_mf/ThermoMechaIGA/pysrc/lib/base_functions.py:583-670)."""
    r = wq_rules.wq_rule(p, nel)
    tag = f"p{p}_n{nel}"
    np.testing.assert_allclose(r["x"], golden[f"{tag}_x"], rtol=0, atol=1e-15)
    for k in KEYS:
        assert _rel(r[k], golden[f"{tag}_{k}"]) < RULE_TOL, k


@pytest.mark.parametrize("p,nel", [(2, 4), (3, 5), (3, 12), (4, 6), (4, 15)])
def test_rule_reproduces_exact_integrals(p, nel):
    """sum_q W[i,q] B[j,q] equals the exact integral for every pair of
    B-splines (the defining property, base_functions.py:469-479)."""
    r = wq_rules.wq_rule(p, nel)
    I = wq_rules.exact_integrals(p, nel)
    for (w, b, key) in (("W00", "B0", "00"), ("W01", "B1", "01"),
                        ("W10", "B0", "10"), ("W11", "B1", "11")):
        got = r[w] @ r[b].T
        assert _rel(got, I[key]) < 1e-12, key


@pytest.mark.parametrize("p,nel", CASES + [(3, 64), (4, 32)])
def test_library_rule_matches_oracle(p, nel):
    from yeti_b200 import _lib
    L = _lib.lib()
    nf, nq = p + nel, 2 * (p + nel) - 1
    arrs = [np.zeros(nq)] + [np.zeros((nf, nq)) for _ in KEYS]
    _lib.check(L.yeti_wq_rule_1d(p, nel, *[a.ctypes.data for a in arrs]),
               "yeti_wq_rule_1d")
    r = wq_rules.wq_rule(p, nel)
    np.testing.assert_allclose(arrs[0], r["x"], rtol=0, atol=1e-15)
    for a, k in zip(arrs[1:], KEYS):
        assert _rel(a, r[k]) < RULE_TOL, k


def test_library_rule_cache_returns_the_computed_rule():
    """The library keeps the rules of the (p, nel) it has built; a rule
    served from that cache is the computed one bit for bit, in any order of
    requests."""
    from yeti_b200 import _lib
    L = _lib.lib()

    def rule(p, nel):
        nf, nq = p + nel, 2 * (p + nel) - 1
        arrs = [np.zeros(nq)] + [np.zeros((nf, nq)) for _ in KEYS]
        _lib.check(L.yeti_wq_rule_1d(p, nel, *[a.ctypes.data for a in arrs]),
                   "yeti_wq_rule_1d")
        return arrs
    seq = [(2, 37), (3, 41), (2, 37), (4, 29), (3, 41), (2, 37)]
    first = {}
    for p, nel in seq:
        got = rule(p, nel)
        if (p, nel) in first:
            for a, b in zip(got, first[(p, nel)]):
                assert a.tobytes() == b.tobytes()
        else:
            first[(p, nel)] = got


def test_library_rule_rejects_bad_sizes():
    from yeti_b200 import _lib
    L = _lib.lib()
    assert L.yeti_wq_rule_1d_size(3, 1, None, None) == -1
    assert L.yeti_wq_rule_1d_size(0, 4, None, None) == -1
