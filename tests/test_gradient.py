"""Adjoint compliance shape gradient: oracle vs finite differences (CPU) and
GPU kernel vs oracle (bit-identical) and vs finite differences.

The reference's own pin (benchs/grad_solid/test_grad_solid_unit_cube_centrif.py)
asserts AN == FD within rtol 1e-5 on the p=1 unit cube under a centrifugal
load; the bar here is 1e-6 relative to central FD (h = 1e-6).
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle
from conftest import load_fixture


def _oracle_compliance(d, args, coords):
    a = list(args)
    a[2] = coords
    k, r, c, F = oracle.sys_linmat_lindef_static(*a)
    n = int(d["nb_dof_tot"])
    K = sp.coo_matrix((k, (r, c)), shape=(n, n)).tocsc()
    K = K + K.T
    idof = d["ind_dof_free"][:int(d["nb_dof_free"])] - 1
    U = np.zeros(n)
    U[idof] = spla.spsolve(K[idof, :][:, idof], F[idof])
    return 0.5 * U @ F, U


def _fd(fun, X0, sel, h=1e-6):
    out = []
    for cp in sel:
        for c in range(3):
            Xp, Xm = X0.copy(), X0.copy()
            Xp[c, cp] += h
            Xm[c, cp] -= h
            out.append((fun(Xp) - fun(Xm)) / (2 * h))
    return np.array(out)


# ---------------------------------------------------------------------- CPU
def test_oracle_gradient_unit_cube_centrifugal_vs_fd():
    """The reference's own gradient case (centrifugal body load, U101)."""
    d, args = load_fixture("grad_unit_cube")
    X0 = np.array(d["COORDS3D"], dtype=float)
    C0, U = _oracle_compliance(d, args, X0)
    sol = U.reshape(-1, 3).T
    gi, ge = oracle.grad_lin_elast_work(args, sol, 0.5 * sol[None])
    g = gi[0] + 2 * ge[0]
    sel = np.arange(X0.shape[1])
    fd = _fd(lambda X: _oracle_compliance(d, args, X)[0], X0, sel)
    an = np.array([g[c, cp] for cp in sel for c in range(3)])
    np.testing.assert_allclose(an, fd, rtol=1e-5, atol=1e-8 * np.abs(fd).max())


def test_oracle_gradient_with_traction_term_vs_fd():
    """Outward pressure on the annulus: the surface-load sensitivity (absent
    from the reference) makes AN agree with FD; without it, it does not."""
    d, args = load_fixture("quarter_annulus_p2_4x4x2")
    X0 = np.array(d["COORDS3D"], dtype=float)
    C0, U = _oracle_compliance(d, args, X0)
    sol = U.reshape(-1, 3).T
    rng = np.random.default_rng(0)
    sel = rng.choice(X0.shape[1], size=8, replace=False)
    fd = _fd(lambda X: _oracle_compliance(d, args, X)[0], X0, sel)
    gi, ge = oracle.grad_lin_elast_work(args, sol, 0.5 * sol[None], include_surface=True)
    g = gi[0] + 2 * ge[0]
    an = np.array([g[c, cp] for cp in sel for c in range(3)])
    assert np.linalg.norm(an - fd) / np.linalg.norm(fd) < 1e-6
    gi, ge = oracle.grad_lin_elast_work(args, sol, 0.5 * sol[None], include_surface=False)
    g = gi[0] + 2 * ge[0]
    an = np.array([g[c, cp] for cp in sel for c in range(3)])
    assert np.linalg.norm(an - fd) / np.linalg.norm(fd) > 0.1


# ---------------------------------------------------------------------- GPU
GRAD_CASES = ["grad_unit_cube", "quarter_annulus_p2_4x4x2", "dload_beam_dist",
              "cantilever_p2_16x4x4", "volume_force_3d"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", GRAD_CASES)
@pytest.mark.parametrize("surface", [False, True])
def test_gpu_gradient_matches_oracle(cuda_ok, name, surface):
    from yeti_b200.gradient import grad_from_system_args
    d, args = load_fixture(name)
    X0 = np.array(d["COORDS3D"], dtype=float)
    rng = np.random.default_rng(1)
    sol = rng.standard_normal((3, X0.shape[1]))
    adj = rng.standard_normal((2, 3, X0.shape[1]))
    gi0, ge0 = oracle.grad_lin_elast_work(args, sol, adj, include_surface=surface)
    gi1, ge1 = grad_from_system_args(args, sol, adj, True, True, surface)
    # same operation order, no FMA contraction: bit-identical
    np.testing.assert_array_equal(gi1, gi0)
    np.testing.assert_array_equal(ge1, ge0)


@pytest.mark.gpu
def test_gpu_autograd_compliance_backward(cuda_ok):
    import torch
    from yeti_b200.gradient import Compliance, compliance_and_gradient
    d, args = load_fixture("quarter_annulus_p2_4x4x2")
    X = torch.tensor(np.array(d["COORDS3D"], dtype=float), requires_grad=True)
    C = Compliance.apply(X, args)
    C.backward()
    C0, g0 = compliance_and_gradient(args)
    assert abs(C.item() - C0) <= 1e-14 * abs(C0)
    np.testing.assert_array_equal(X.grad.numpy(), g0)


@pytest.mark.gpu
def test_gpu_gradient_annulus_32x32x2_vs_fd(cuda_ok):
    """Quarter annulus (R 1 -> 4, t 0.1, exact arcs), p=2, 32x32x2 elements,
    outward unit pressure on the outer face: AN (GPU, with the traction term)
    vs central FD (h=1e-6) on 20 seeded control points x 3 coordinates."""
    from yeti_b200.gradient import compliance_and_gradient
    d, args = load_fixture("quarter_annulus_p2_32x32x2")
    X0 = np.array(d["COORDS3D"], dtype=float)
    C0, g = compliance_and_gradient(args)
    rng = np.random.default_rng(20)
    sel = rng.choice(X0.shape[1], size=20, replace=False)
    fd = _fd(lambda X: _gpu_compliance(args, X), X0, sel)
    an = np.array([g[c, cp] for cp in sel for c in range(3)])
    assert np.linalg.norm(an - fd) / np.linalg.norm(fd) < 1e-6


def _gpu_compliance(args, X):
    from yeti_b200.gradient import _solve
    U, F = _solve(args, X)
    return 0.5 * U @ F


# ------------------------------------------- degrees beyond 2 (synthetic)
# (degrees, elements, load 'U2<type>' on the face u = 1 with its magnitude)
HIGH = [(4, (2, 1, 1), (3, -1.0)), ((3, 2, 4), (2, 2, 1), (0, 1.0))]


def _high_args(p, nel, load):
    from yeti_b200.patches import cube_patch, u1_system_args
    P = cube_patch(nel, p, size=(2.0, 1.0, 1.0), perturb=0.1, wrange=(0.9, 1.1), seed=9)
    return u1_system_args(P, E=100.0, nu=0.3, clamp_u0=True, load_u1=load)


@pytest.mark.parametrize("p,nel,load", HIGH)
def test_oracle_gradient_high_degree_with_traction_vs_fd(p, nel, load):
    """p=4 and mixed degrees (3,2,4), clamped face u=0, a fixed-direction
    traction / a normal pressure on the face u=1: AN with the surface term
    vs central FD on 8 seeded control points x 3 coordinates."""
    from yeti_b200.stiffmtrx_elemstorage import SYSTEM_ARG_NAMES
    args = _high_args(p, nel, load)
    d = dict(zip(SYSTEM_ARG_NAMES, args))
    X0 = np.asarray(args[2], dtype=float)
    C0, U = _oracle_compliance(d, args, X0)
    sol = U.reshape(-1, 3).T
    gi, ge = oracle.grad_lin_elast_work(args, sol, 0.5 * sol[None], include_surface=True)
    g = gi[0] + 2.0 * ge[0]
    sel = np.random.default_rng(3).choice(X0.shape[1], size=8, replace=False)
    fd = _fd(lambda X: _oracle_compliance(d, args, X)[0], X0, sel)
    an = np.array([g[c, cp] for cp in sel for c in range(3)])
    assert np.linalg.norm(an - fd) / np.linalg.norm(fd) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("p,nel,load", HIGH)
def test_gpu_gradient_high_degree_vs_fd_and_oracle(cuda_ok, p, nel, load):
    from yeti_b200.gradient import compliance_and_gradient, grad_from_system_args
    args = _high_args(p, nel, load)
    X0 = np.asarray(args[2], dtype=float)
    C0, g = compliance_and_gradient(args)
    sel = np.random.default_rng(3).choice(X0.shape[1], size=8, replace=False)
    fd = _fd(lambda X: _gpu_compliance(args, X), X0, sel)
    an = np.array([g[c, cp] for cp in sel for c in range(3)])
    assert np.linalg.norm(an - fd) / np.linalg.norm(fd) < 1e-6
    # and the kernel equals the oracle bit for bit on the same state
    rng = np.random.default_rng(4)
    sol = rng.standard_normal((3, X0.shape[1]))
    adj = rng.standard_normal((2, 3, X0.shape[1]))
    gi, ge = grad_from_system_args(args, sol, adj, include_surface=True)
    oi, oe = oracle.grad_lin_elast_work(args, sol, adj, include_surface=True)
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(ge, oe)
