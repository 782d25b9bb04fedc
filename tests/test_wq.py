"""Weighted-quadrature elasticity: oracle properties (CPU) and GPU parity.

Bars: FP64 apply / diagonal / body force within 1e-12 relative (2-norm) of
the FP64 oracle; FP32 apply within 2e-6; the FP64 PCG solution within 1e-9
of the oracle's direct solve at rtol 1e-11; the mixed-precision solve within
1e-7 of the FP64 one at rtol 1e-8.
"""
import numpy as np
import pytest

from oracle.wq_ops import WQOracle
from yeti_b200.patches import cube_patch, free_mask

CASES = [
    # (nel, p, perturb, wrange, clamp)
    ((2, 3, 2), (2, 2, 2), 0.0, None, None),
    ((3, 4, 5), (2, 3, 2), 0.2, (0.8, 1.2), {"w0": (0, 1, 2)}),
    ((7, 3, 4), (3, 3, 3), 0.2, (0.8, 1.2), {"w0": (0, 1, 2)}),
    ((9, 8, 6), (3, 2, 4), 0.15, (0.9, 1.1), {"u0": (0,), "v1": (1, 2)}),
    ((5, 11, 3), (4, 3, 2), 0.1, (0.8, 1.2), {"w0": (0, 1, 2), "w1": (2,)}),
]
# One degree in all directions (2..5) runs the streaming apply kernel: cases
# with several (u, v) tiles and element ranges.
STREAM_CASES = [
    ((17, 12, 6), (3, 3, 3), 0.2, (0.8, 1.2), {"w0": (0, 1, 2)}),
    ((20, 9, 5), (2, 2, 2), 0.1, (0.9, 1.1), {"w1": (0, 1, 2)}),
    ((12, 11, 5), (4, 4, 4), 0.15, (0.8, 1.2), {"u0": (0,), "v1": (1, 2)}),
    ((6, 18, 9), (5, 5, 5), 0.1, None, None),
    ((10, 24, 4), (3, 3, 3), 0.2, (0.8, 1.2), {"v0": (0, 1, 2)}),
]

# Thin patches (two elements, the fewest the WQ rule takes): tiles that are
# first and last at once, one tile along u with many along v and back.
THIN_CASES = [
    ((2, 2, 2), (2, 2, 2), 0.1, (0.9, 1.1), None),
    ((2, 3, 2), (3, 3, 3), 0.1, (0.9, 1.1), {"w0": (0, 1, 2)}),
    ((2, 2, 5), (4, 4, 4), 0.1, (0.9, 1.1), None),
    ((16, 2, 2), (2, 2, 2), 0.1, (0.9, 1.1), {"u0": (0, 1, 2)}),
    ((2, 17, 2), (3, 3, 3), 0.1, (0.9, 1.1), None),
    ((33, 2, 2), (2, 2, 2), 0.1, (0.9, 1.1), {"v1": (1,)}),
    ((3, 2, 2), (5, 5, 5), 0.1, (0.9, 1.1), None),
]


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


# ---------------------------------------------------------------------- CPU
def test_oracle_affine_unit_weights_is_symmetric_and_exact():
    """On an affine patch with unit weights the WQ rules are exact: the
    operator is symmetric and annihilates rigid-body motions."""
    P = cube_patch((3, 3, 3), (2, 2, 2), size=(2.0, 1.0, 1.5))
    K = WQOracle(P, 1.0, 0.3).matrix()
    s = np.abs(K).max()
    assert np.abs(K - K.T).max() < 1e-13 * s
    X = P["cps"]
    for c in range(3):
        m = np.zeros_like(X)
        m[c] = 1.0
        assert np.abs(K @ m.ravel()).max() < 1e-13 * s
    m = np.zeros_like(X)
    m[0], m[1] = -X[1], X[0]
    assert np.abs(K @ m.ravel()).max() < 1e-13 * s


def test_oracle_pcg_matches_direct_solve():
    P = cube_patch((3, 3, 3), (3, 3, 3), perturb=0.2, wrange=(0.8, 1.2), seed=2)
    clamp = {"w0": (0, 1, 2)}
    op = WQOracle(P, 1.0, 0.3, clamp)
    b = op.body_force([0.0, 0.0, -1.0])
    x, it, res = op.pcg(b, rtol=1e-11)
    m = free_mask(P, clamp) > 0
    K = op.matrix()
    xd = np.zeros_like(b)
    xd[m] = np.linalg.solve(K[np.ix_(m, m)], b[m])
    assert res < 1e-11 and _rel(x, xd) < 1e-9


def test_oracle_diag_matches_matrix_diagonal():
    P = cube_patch((3, 2, 3), (3, 2, 2), perturb=0.2, wrange=(0.8, 1.2), seed=4)
    op = WQOracle(P, 2.0, 0.25, {"u0": (0, 1)})
    K = op.matrix()
    d = op.diag()
    m = op.mask.ravel() > 0
    assert np.abs(d[m] - np.diag(K)[m]).max() < 1e-13 * np.abs(np.diag(K)).max()


# ---------------------------------------------------------------------- GPU
def _pair(case, E=1.0, nu=0.3, seed=7):
    from yeti_b200.wq import WQElasticity
    nel, p, pert, wr, clamp = case
    P = cube_patch(nel, p, perturb=pert, wrange=wr, seed=seed)
    return WQElasticity(P, E, nu, clamp), WQOracle(P, E, nu, clamp)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES + STREAM_CASES + THIN_CASES)
def test_gpu_apply_diag_force_match_oracle(cuda_ok, case):
    op, ref = _pair(case)
    rng = np.random.default_rng(11)
    u = rng.standard_normal(op.ndof)
    k0 = ref.apply(u)
    k1 = op.eval_Ku(u)
    assert _rel(k1, k0) < 1e-12
    k2 = op.eval_Ku(u.astype(np.float32), precision="f32")
    assert k2.dtype == np.float32
    assert _rel(k2.astype(np.float64), k0) < 2e-6
    assert _rel(op.diag(), ref.diag()) < 1e-12
    f0 = ref.body_force([0.3, -0.2, -1.0])
    f1 = op.eval_bodyforce_vector([0.3, -0.2, -1.0])
    assert _rel(f1, f0) < 1e-12
    # clamped dofs: zero output whatever the input
    m = op.free_mask == 0
    if m.any():
        assert np.abs(k1[m]).max() == 0.0


@pytest.mark.gpu
def test_gpu_setup_rejects_a_single_element_direction(cuda_ok):
    from yeti_b200._lib import YetiError
    from yeti_b200.wq import WQElasticity
    P = cube_patch((1, 3, 2), (2, 2, 2))
    with pytest.raises(YetiError, match="EINVAL"):
        WQElasticity(P, 1.0, 0.3, None)


@pytest.mark.gpu
def test_gpu_pcg_fp64_and_mixed_match_direct(cuda_ok):
    case = ((4, 4, 4), (3, 3, 3), 0.2, (0.8, 1.2), {"w0": (0, 1, 2)})
    op, ref = _pair(case, seed=3)
    b = ref.body_force([0.0, 0.0, -1.0])
    m = op.free_mask > 0
    K = ref.matrix()
    xd = np.zeros_like(b)
    xd[m] = np.linalg.solve(K[np.ix_(m, m)], b[m])
    x64, st = op.pcg(b, rtol=1e-11)
    assert st["status"] == 0 and st["rel_residual"] <= 1e-11
    assert _rel(x64, xd) < 1e-9
    x32, st32 = op.pcg(b, rtol=1e-8, mixed=True)
    assert st32["status"] == 0 and st32["rel_residual"] <= 1e-8
    assert st32["fp32_applies"] > 0 and st32["outer_iterations"] >= 1
    assert _rel(x32, xd) < 1e-7
    for mixed in (False, True):
        xb, stb = op.pcg(b, rtol=1e-10, mixed=mixed, method="bicgstab")
        assert stb["status"] == 0 and stb["rel_residual"] <= 1e-10
        assert _rel(xb, xd) < 1e-8


@pytest.mark.gpu
def test_gpu_apply_device_tensors_and_linearity(cuda_ok):
    import torch
    case = ((12, 10, 8), (3, 3, 3), 0.2, (0.8, 1.2), {"w0": (0, 1, 2)})
    op, _ = _pair(case)
    g = torch.Generator(device="cuda").manual_seed(0)
    u = torch.randn(op.ndof, dtype=torch.float64, device="cuda", generator=g)
    v = torch.randn(op.ndof, dtype=torch.float64, device="cuda", generator=g)
    ku, kv = op.eval_Ku(u), op.eval_Ku(v)
    kw = op.eval_Ku(2.5 * u - 0.75 * v)
    lin = (2.5 * ku - 0.75 * kv)
    assert (torch.linalg.norm(kw - lin) / torch.linalg.norm(lin)).item() < 1e-13
    # FP32 apply agrees with FP64 to single precision
    k32 = op.eval_Ku(u.float(), precision="f32").double()
    assert (torch.linalg.norm(k32 - ku) / torch.linalg.norm(ku)).item() < 2e-6


@pytest.mark.parametrize("case", CASES[1:4])
def test_reference_algorithm_cpu_matches_oracle(case):
    """oracle/oracle_wq.c (the reference's rank-one sparse products, used as
    the timed CPU baseline) computes the same operator as the numpy oracle."""
    from oracle.wq_cpu import ReferenceWQ
    nel, p, pert, wr, clamp = case
    P = cube_patch(nel, p, perturb=pert, wrange=wr, seed=5)
    a = WQOracle(P, 1.0, 0.3, clamp)
    b = ReferenceWQ(P, 1.0, 0.3, clamp)
    u = np.random.default_rng(1).standard_normal(a.ndof)
    assert _rel(b.apply(u), a.apply(u)) < 1e-13


@pytest.mark.parametrize("case", CASES[1:4])
def test_reference_algorithm_cpu_diagonal_and_cg_loop(case):
    """The timed CPU baseline's diagonal (find_physical_diag_3d per diagonal
    block) and its Jacobi-PCG loop (wq_mf_cg_3d's iteration with z = r/diag)
    reproduce the numpy oracle's diagonal and its PCG iterate after the same
    number of iterations."""
    from oracle.wq_cpu import ReferenceWQ
    nel, p, pert, wr, clamp = case
    P = cube_patch(nel, p, perturb=pert, wrange=wr, seed=5)
    a = WQOracle(P, 1.0, 0.3, clamp)
    b = ReferenceWQ(P, 1.0, 0.3, clamp)
    d = b.diag()
    assert _rel(d, a.diag()) < 1e-13
    rhs = a.body_force([0.0, 0.0, -1.0])
    t, x, rel = b.pcg_seconds(rhs, d, 7)
    x0, it, _ = a.pcg(rhs, rtol=1e-300, maxit=7)
    assert it == 7 and t > 0
    assert _rel(x, x0) < 1e-10
    assert np.isfinite(rel) and rel > 0


def test_reference_algorithm_cpu_declares_pointers():
    """Large arrays can live at addresses beyond 32 bits (the bench's CPU
    baseline runs the C port on the 64^3 workload): every pointer argument of
    the port is declared, so ctypes passes full addresses; a patch with
    arrays of a few hundred KB still matches the numpy oracle."""
    import ctypes
    from oracle.wq_cpu import ReferenceWQ
    P = cube_patch((22, 20, 16), 2, perturb=0.1, wrange=(0.9, 1.1), seed=6)
    a = WQOracle(P, 1.0, 0.3, {"w0": (0, 1, 2)})
    b = ReferenceWQ(P, 1.0, 0.3, {"w0": (0, 1, 2)})
    for f in (b.L.oracle_wq_create, b.L.oracle_wq_apply, b.L.oracle_wq_free,
              b.L.oracle_wq_diag, b.L.oracle_wq_pcg_seconds):
        assert f.argtypes is not None
        assert all(t in (ctypes.c_void_p, ctypes.c_double, ctypes.c_int) for t in f.argtypes)
    u = np.random.default_rng(2).standard_normal(a.ndof)
    assert _rel(b.apply(u), a.apply(u)) < 1e-13
