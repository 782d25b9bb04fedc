"""The WQ operator pinned to the reference's own Python WQ assembly.

tests/golden/wq_operator.npz holds products K X computed by the reference's
``methods_wq.WQ.eval_conductivity_matrix`` (methods_wq.py:76-108) from its
own 1-D rules and Jacobian (create_model.py:531-601), made by
tests/golden/make_wq_operator_golden.py:

* box_*/sym_*: the elastic operator, block (a, b) assembled with the
  Fortran's coefficient S[(a,k),(b,l)] (eval_mech_coefficient,
  wq_assembly.f90:52-138), on an axis-aligned box and on maps x = grad(phi)
  (symmetric Jacobians, where the Fortran's coefficient orientation equals
  the geometric one);
* gen_*: perturbed patches: the Jacobian, the scalar conductivity
  coefficient inv(J) inv(J)^T det(J) and the scalar operator.

CPU tests check the oracle against them (1e-12 relative); GPU tests check
the library's FP64 apply against them directly (1e-12) and its FP32 apply
(2e-6, the FP32 tolerance of the other WQ tests).
"""
import numpy as np
import pytest

from conftest import ROOT

GOLD = np.load(f"{ROOT}/tests/golden/wq_operator.npz")
ELASTIC = ["box_p4", "sym_p2", "sym_p3", "sym_p2_long"]
GENERAL = ["gen_p2", "gen_p3"]


def _patch(name):
    p = tuple(int(v) for v in GOLD[f"{name}_p"])
    nel = tuple(int(v) for v in GOLD[f"{name}_nel"])
    cps = np.ascontiguousarray(GOLD[f"{name}_cps"])
    return {"p": p, "nel": nel, "cps": cps, "weights": np.ones(cps.shape[1])}


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _oracle(name):
    from oracle.wq_ops import WQOracle
    return WQOracle(_patch(name), 1.0, 0.3)


@pytest.mark.parametrize("name", ELASTIC + GENERAL)
def test_oracle_jacobian_matches_reference(name):
    o = _oracle(name)
    J = GOLD[f"{name}_J"]
    assert _rel(o.J.reshape(3, 3, -1), J) < 1e-12


@pytest.mark.parametrize("name", ELASTIC)
def test_oracle_elastic_operator_matches_reference(name):
    o = _oracle(name)
    X, KX = GOLD[f"{name}_X"], GOLD[f"{name}_KX"]
    for k in range(X.shape[1]):
        assert _rel(o.apply(X[:, k]), KX[:, k]) < 1e-12, k


@pytest.mark.parametrize("name", GENERAL)
def test_oracle_scalar_operator_matches_reference(name):
    o = _oracle(name)
    C = o.conductivity_coef()
    assert _rel(C, GOLD[f"{name}_kcoef"]) < 1e-12
    X, KX = GOLD[f"{name}_X"], GOLD[f"{name}_KX"]
    for k in range(X.shape[1]):
        assert _rel(o.apply_scalar(X[:, k], C), KX[:, k]) < 1e-12, k


def test_planted_coefficient_error_is_caught():
    """The pin is sharp: the oracle with its coefficient transposed per 3x3
    block (a mistake planted on the CPU) misses the reference's product on
    the curved symmetric map by far more than the tolerance."""
    o = _oracle("sym_p3")
    X, KX = GOLD["sym_p3_X"], GOLD["sym_p3_KX"]
    S = o.S.copy()
    for a in range(3):
        for b in range(3):
            blk = S[..., 3 * a:3 * a + 3, 3 * b:3 * b + 3]
            S[..., 3 * a:3 * a + 3, 3 * b:3 * b + 3] = np.swapaxes(blk, -1, -2)
    o.S = S
    assert _rel(o.apply(X[:, 0]), KX[:, 0]) > 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("name", ELASTIC)
def test_gpu_apply_matches_reference_operator(cuda_ok, name):
    from yeti_b200.wq import WQElasticity
    op = WQElasticity(_patch(name), 1.0, 0.3, precisions="both")
    X, KX = GOLD[f"{name}_X"], GOLD[f"{name}_KX"]
    for k in range(X.shape[1]):
        assert _rel(op.eval_Ku(X[:, k]), KX[:, k]) < 1e-12, k
        k32 = op.eval_Ku(X[:, k].astype(np.float32), precision="f32")
        assert _rel(k32.astype(np.float64), KX[:, k]) < 2e-6, k
