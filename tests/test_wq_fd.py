"""Fast-diagonalisation (FD) preconditioner of the WQ elasticity operator
(wq_mf_cg_3d's FD branch, mf_wq_solver.f90:803-953, per displacement
component).

Bars: the oracle's FD inverts the separable operator it is built from to
1e-12; the GPU FD apply matches the oracle within 1e-10 (FP64) / 1e-5 (FP32)
relative; FD-preconditioned CG and BiCGSTAB reach the oracle's direct
solution within 1e-9 (FP64, rtol 1e-11) and the mixed solve within 1e-7 of
the FP64 one (rtol 1e-8), in fewer iterations than Jacobi.
"""
import numpy as np
import pytest

from oracle.wq_ops import WQOracle
from yeti_b200.patches import cube_patch, free_mask

CASES = [
    # (nel, p, perturb, wrange, clamp)
    ((5, 4, 3), (3, 2, 2), 0.2, (0.8, 1.2), {"w0": (0, 1, 2), "u1": (0,)}),
    ((9, 8, 6), (3, 2, 4), 0.15, (0.9, 1.1), {"u0": (0,), "v1": (1, 2), "w0": (0,)}),
    ((12, 11, 5), (4, 4, 4), 0.15, (0.8, 1.2), {"w0": (0, 1, 2), "w1": (2,)}),
    ((17, 12, 6), (3, 3, 3), 0.2, (0.8, 1.2), {"w0": (0, 1, 2)}),
]
VARIANTS = [("fd", False, False, False), ("fd_scaled", True, False, False),
            ("fd_unit", False, True, False), ("fd_td", False, False, True),
            ("fd_td_scaled", True, False, True)]


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _patch(case, seed=7):
    nel, p, pert, wr, clamp = case
    return cube_patch(nel, p, perturb=pert, wrange=wr, seed=seed), clamp


# ---------------------------------------------------------------------- CPU
@pytest.mark.parametrize("unit", [False, True])
def test_oracle_fd_inverts_its_separable_operator(unit):
    P, clamp = _patch(CASES[0])
    op = WQOracle(P, 1.0, 0.3, clamp)
    plan = op.fd_setup(scaled=False, unit=unit)
    rng = np.random.default_rng(1)
    for c, pc in enumerate(plan):
        (Ku, Mu), (Kv, Mv), (Kw, Mw) = [op.fd_1d(d, *pc["box"][d]) for d in range(3)]
        a = pc["a"]
        Pc = (a[0] * np.kron(Mw, np.kron(Mv, Ku)) + a[1] * np.kron(Mw, np.kron(Kv, Mu))
              + a[2] * np.kron(Kw, np.kron(Mv, Mu)))
        sl = tuple(slice(*pc["box"][d]) for d in (2, 1, 0))
        r = np.zeros(op.mask.shape)
        x = rng.standard_normal(r[c][sl].shape)
        r[c][sl] = (Pc @ x.ravel()).reshape(x.shape)
        z = op.fd_apply(r.ravel(), plan).reshape(op.mask.shape)
        assert np.abs(z[c][sl] - x).max() < 1e-12 * np.abs(x).max()
        others = [k for k in range(3) if k != c]
        assert all(np.abs(z[k]).max() == 0.0 for k in others)


def test_oracle_td_weights_of_a_constant_coefficient():
    """On an affine box with unit weights the diagonal coefficients are
    constant; the tensor decomposition then returns constant weights whose
    products reproduce them: K_k M_l M_m = S[(c,k),(c,k)] for {k, l, m} the
    three directions."""
    P = cube_patch((4, 3, 5), (2, 2, 2), size=(2.0, 1.0, 1.5))
    op = WQOracle(P, 1.0, 0.3, {"w0": (0, 1, 2)})
    for c in range(3):
        M, K = op.td_weights(c)
        for k in range(3):
            cc = op.S[..., 3 * c + k, 3 * c + k]
            assert np.ptp(cc) < 1e-12 * np.abs(cc).max()
            others = [d for d in range(3) if d != k]
            prod = K[k] * M[others[0]].mean() * M[others[1]].mean()
            assert np.abs(prod - cc.mean()).max() < 1e-10 * cc.mean()
            assert np.ptp(K[k]) < 1e-10 * K[k].mean()


def test_oracle_fd_pcg_matches_direct_solve_in_fewer_iterations():
    P, clamp = _patch(CASES[0])
    op = WQOracle(P, 1.0, 0.3, clamp)
    b = op.body_force([0.0, 0.0, -1.0])
    m = free_mask(P, clamp) > 0
    K = op.matrix()
    xd = np.zeros_like(b)
    xd[m] = np.linalg.solve(K[np.ix_(m, m)], b[m])
    _, it_j, _ = op.pcg(b, rtol=1e-11)
    for name, scaled, unit, td in VARIANTS:
        plan = op.fd_setup(scaled, unit, td)
        x, it, res = op.pcg(b, rtol=1e-11, precond=lambda v: op.fd_apply(v, plan))
        assert res < 1e-11 and _rel(x, xd) < 1e-9, name
        assert it < it_j, (name, it, it_j)


# ---------------------------------------------------------------------- GPU
def _pair(case, E=1.0, nu=0.3, seed=7):
    from yeti_b200.wq import WQElasticity
    P, clamp = _patch(case, seed)
    return WQElasticity(P, E, nu, clamp), WQOracle(P, E, nu, clamp)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("variant", VARIANTS, ids=[v[0] for v in VARIANTS])
def test_fd_apply_matches_oracle(cuda_ok, case, variant):
    from yeti_b200._lib import PREC_F32, PREC_F64
    name, scaled, unit, td = variant
    gpu, ora = _pair(case)
    plan = ora.fd_setup(scaled, unit, td)
    r = np.random.default_rng(3).standard_normal(ora.ndof) * ora.mask.ravel()
    z_ref = ora.fd_apply(r, plan)
    z64 = gpu.fd_apply(r, name, PREC_F64)
    assert _rel(z64, z_ref) < 1e-10
    assert np.all(z64[ora.mask.ravel() == 0] == 0.0)
    z32 = gpu.fd_apply(r.astype(np.float32), name, PREC_F32)
    assert _rel(z32.astype(np.float64), z_ref) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("variant", VARIANTS, ids=[v[0] for v in VARIANTS])
@pytest.mark.parametrize("method", ["cg", "bicgstab"])
def test_fd_pcg_reaches_direct_solution(cuda_ok, variant, method):
    name = variant[0]
    case = CASES[0]
    gpu, ora = _pair(case)
    P, clamp = _patch(case)
    b = ora.body_force([0.0, 0.0, -1.0])
    m = free_mask(P, clamp) > 0
    K = ora.matrix()
    xd = np.zeros_like(b)
    xd[m] = np.linalg.solve(K[np.ix_(m, m)], b[m])
    x, st = gpu.pcg(b, rtol=1e-11, method=method, precond=name)
    assert st["rel_residual"] <= 1e-11 and _rel(x, xd) < 1e-9
    _, st_j = gpu.pcg(b, rtol=1e-11, method=method)
    assert st["iterations"] < st_j["iterations"]
    xm, stm = gpu.pcg(b, rtol=1e-8, method=method, precond=name, mixed=True)
    assert stm["rel_residual"] <= 1e-8 and _rel(xm, x) < 1e-7
    assert stm["fp32_applies"] > 0


@pytest.mark.gpu
def test_fd_pcg_larger_patch_cuts_iterations(cuda_ok):
    """On a 24^3 p=3 patch (the streaming apply) FD-preconditioned CG needs
    a fraction of Jacobi's iterations, FP64 and mixed."""
    from yeti_b200.wq import WQElasticity
    P = cube_patch((24, 24, 24), (3, 3, 3), perturb=0.2, wrange=(0.8, 1.2), seed=11)
    clamp = {"w0": (0, 1, 2)}
    op = WQElasticity(P, 1.0, 0.3, clamp)
    b = op.eval_bodyforce_vector([0.0, 0.0, -1.0])
    xj, stj = op.pcg(b, rtol=1e-9)
    for mixed in (False, True):
        x, st = op.pcg(b, rtol=1e-9, mixed=mixed, precond="fd_scaled")
        assert st["rel_residual"] <= 1e-9
        assert _rel(x, xj) < 1e-7
        assert 3 * st["iterations"] < stj["iterations"], (st["iterations"], stj["iterations"])


@pytest.mark.gpu
@pytest.mark.parametrize("nel,p,size", [((64, 64, 64), 3, (1.0, 1.0, 1.0)),
                                        ((128, 128, 32), 4, (4.0, 4.0, 1.0))])
def test_fd_benchmark_sizes(cuda_ok, nel, p, size):
    """The tile shapes of the benchmark patches (shared-memory tiles above
    48 KB, two row tiles for 132 functions): FP32 and FP64 applications agree,
    the FP64 one is symmetric, and mixed FD-preconditioned CG converges in
    under 60 iterations."""
    from yeti_b200._lib import PREC_F32, PREC_F64
    from yeti_b200.wq import WQElasticity
    P = cube_patch(nel, p, size=size, perturb=0.1, wrange=(0.8, 1.2), seed=5)
    op = WQElasticity(P, 1.0, 0.3, {"w0": (0, 1, 2)})
    rng = np.random.default_rng(2)
    x, y = rng.standard_normal(op.ndof), rng.standard_normal(op.ndof)
    zx = op.fd_apply(x, "fd", PREC_F64)
    zy = op.fd_apply(y, "fd", PREC_F64)
    assert abs(y @ zx - x @ zy) < 1e-12 * abs(y @ zx)
    z32 = op.fd_apply(x.astype(np.float32), "fd", PREC_F32).astype(np.float64)
    assert _rel(z32, zx) < 1e-5
    b = op.eval_bodyforce_vector([0.0, 0.0, -1.0])
    xs, st = op.pcg(b, rtol=1e-8, mixed=True, precond="fd")
    assert st["rel_residual"] <= 1e-8 and st["iterations"] < 60


@pytest.mark.gpu
def test_fd_rejects_unclamped_component(cuda_ok):
    """A component with no clamped face makes its separable operator
    singular: the library refuses instead of dividing by a zero eigenvalue."""
    from yeti_b200._lib import YetiError
    from yeti_b200.wq import WQElasticity
    P = cube_patch((4, 4, 4), (2, 2, 2), perturb=0.1, seed=2)
    op = WQElasticity(P, 1.0, 0.3, {"w0": (0, 1)})
    b = op.eval_bodyforce_vector([0.0, 0.0, -1.0])
    with pytest.raises(YetiError, match="no clamped face"):
        op.pcg(b, precond="fd")
    with pytest.raises(ValueError):
        op.pcg(b, precond="tensor")
