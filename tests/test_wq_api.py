"""The reference's WQ Python API shape: WQElasticity.from_iga_model (the
fortran_mf_wq(modelIGA, mechablockedboundaries=...) constructor,
fortran_mf_wq.py:31-71) and mf_conj_grad's RelRes / RelError histories
(fortran_mf_wq.py:545-560, mf_wq_solver.f90:656,697,785-792).

The model is the p=2 16x4x4 cantilever preprocessed by the reference's own
Python (tests/golden/cantilever_p2_16x4x4.npz), handed over as an object
with the IGAparametrization attributes the constructor reads.  The block is
affine with unit weights, where the WQ rules integrate exactly: the WQ
solution must equal the Gauss-quadrature COO solution of the same model to
rounding, which checks the control-point numbering between the two layouts
(the one YETI's VTU writers read).
"""
import types

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle
from conftest import load_fixture
from yeti_b200.patches import clamp_faces_from_blocked, free_mask, patch_from_iga_model

BLOCKED = [[1, 0], [0, 0], [0, 0]]   # clamped face x = 0 (u = 0)


def _model(name="cantilever_p2_16x4x4"):
    d, args = load_fixture(name)
    nkv = d["Nkv"].reshape(3, -1)
    U = d["Ukv"].ravel()
    kv = [U[:nkv[0, 0]], U[nkv[0, 0]:nkv[0, 0] + nkv[1, 0]], U[nkv[0, 0] + nkv[1, 0]:]]
    nel = int(d["nb_elem_patch"].ravel()[0])
    nnode = int(np.asarray(d["NNODE"]).ravel()[0])
    m = types.SimpleNamespace(
        _Jpqr=d["Jpqr"], _Nkv=d["Nkv"], _Ukv=[kv], _COORDS=d["COORDS3D"],
        _nb_cp=int(d["nb_cp"]), _IEN=[d["IEN"].reshape(nel, nnode)], _Nijk=d["Nijk"],
        _weight=list(d["weight"].reshape(nel, nnode)), _elementsByPatch=d["nb_elem_patch"],
        _MATERIAL_PROPERTIES=d["MATERIAL_PROPERTIES"])
    return d, args, m


def _gauss_solution(d, args):
    """COO assembly (oracle) + sparse direct solve of the free dofs."""
    k, r, c, F = oracle.sys_linmat_lindef_static(*args)
    n = F.size
    K = sp.coo_matrix((k, (r, c)), shape=(n, n)).tocsc()
    K = K + K.T
    idof = np.asarray(d["ind_dof_free"]).ravel()[:int(d["nb_dof_free"])] - 1
    U = np.zeros(n)
    U[idof] = spla.spsolve(K[idof, :][:, idof], F[idof])
    return U, F, idof


def _to_tensor(U, cp_index):
    return np.ascontiguousarray(U.reshape(-1, 3).T[:, cp_index]).ravel()


def test_patch_from_iga_model_numbering_and_clamps():
    d, _, m = _model()
    patch, cp = patch_from_iga_model(m)
    assert patch["p"] == (2, 2, 2) and patch["nel"] == (16, 4, 4)
    X = d["COORDS3D"]
    assert np.array_equal(patch["cps"], X[:, cp])
    # the blocked face maps onto the model's own Dirichlet dofs
    mask = free_mask(patch, clamp_faces_from_blocked(BLOCKED)).reshape(3, -1)
    free_model = np.zeros(3 * X.shape[1], dtype=bool)
    free_model[np.asarray(d["ind_dof_free"]).ravel()[:int(d["nb_dof_free"])] - 1] = True
    assert np.array_equal(mask.T[np.argsort(cp)].ravel() > 0, free_model)


def test_wq_oracle_solution_equals_gauss_solution_on_the_model():
    from oracle.wq_ops import WQOracle
    d, args, m = _model()
    patch, cp = patch_from_iga_model(m)
    U, F, idof = _gauss_solution(d, args)
    o = WQOracle(patch, 210000.0, 0.3, clamp_faces_from_blocked(BLOCKED))
    K = o.matrix()
    free = o.mask.ravel() > 0
    f = _to_tensor(F, cp)
    x = np.zeros_like(f)
    x[free] = np.linalg.solve(K[np.ix_(free, free)], f[free])
    u_ref = _to_tensor(U, cp)
    assert np.linalg.norm(x - u_ref) <= 1e-9 * np.linalg.norm(u_ref)
    # a numbering mistake (two control points swapped, planted on the CPU)
    bad = cp.copy()
    bad[[5, 200]] = bad[[200, 5]]
    assert np.linalg.norm(x - _to_tensor(U, bad)) > 1e-3 * np.linalg.norm(u_ref)


@pytest.mark.gpu
def test_from_iga_model_solve_and_model_layout(cuda_ok):
    from yeti_b200.wq import WQElasticity
    d, args, m = _model()
    U, F, idof = _gauss_solution(d, args)
    op = WQElasticity.from_iga_model(m, mechablockedboundaries=BLOCKED)
    f = op.from_model_layout(F)
    x, st = op.pcg(f, rtol=1e-12, maxit=20000)
    Um = op.to_model_layout(x)
    Ug = U.reshape(-1, 3).T
    assert np.linalg.norm(Um - Ug) <= 1e-8 * np.linalg.norm(Ug)


@pytest.mark.gpu
@pytest.mark.parametrize("method,isCG", [("WP", True), ("JM", True), ("WP", False)])
def test_mf_conj_grad_history(cuda_ok, method, isCG):
    """RelRes(0) = 1 and RelRes(k) = max|r_k| / max|b| down to epsilon;
    RelError(k) against a direct solution; the CG history equals a numpy
    Jacobi-CG run with the oracle's operator, iteration by iteration."""
    from oracle.wq_ops import WQOracle
    from yeti_b200.patches import cube_patch
    from yeti_b200.wq import WQElasticity
    P = cube_patch((5, 4, 6), (2, 3, 2), perturb=0.15, wrange=(0.9, 1.1), seed=4)
    clamp = {"w0": (0, 1, 2)}
    op = WQElasticity(P, 1.0, 0.3, clamp)
    o = WQOracle(P, 1.0, 0.3, clamp)
    b = o.body_force([0.0, 0.0, -1.0])
    K = o.matrix()
    free = o.mask.ravel() > 0
    xd = np.zeros_like(b)
    xd[free] = np.linalg.solve(K[np.ix_(free, free)], b[free])
    x, res, err = op.mf_conj_grad(b, 500, 1e-10, method=method, directsol=xd, isCG=isCG)
    assert res[0] == pytest.approx(1.0, rel=1e-12) and err[0] == pytest.approx(1.0, rel=1e-12)
    assert res[-1] <= 1e-10 and np.all(res[:-1] > 1e-10)
    assert err[-1] < 1e-7
    assert np.abs(x - xd).max() / np.abs(xd).max() == pytest.approx(err[-1], rel=1e-6)
    if method == "WP" and isCG:
        dinv = free / o.diag()
        xx = np.zeros_like(b)
        r = b * free
        z = dinv * r
        p = z.copy()
        rz = r @ z
        bmax = np.abs(b * free).max()
        for k in range(1, min(len(res), 40)):
            Ap = o.apply(p)
            a = rz / (p @ Ap)
            xx += a * p
            r -= a * Ap
            assert np.abs(r).max() / bmax == pytest.approx(res[k], rel=1e-6), k
            z = dinv * r
            rzn = r @ z
            p = z + (rzn / rz) * p
            rz = rzn
