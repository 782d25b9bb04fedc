"""Shape-optimisation responses (IgaOptimization, overlay/iga_optimization.py
:69-221, and OPTmodelling's response functions, OPT_modelling.py:411-445,
508-565) on the GPU kernels.

Bars: the responses at x equal the GPU compliance and volume of the moved
model exactly; the analytic gradients (adjoint kernel, volume gradient,
propagated through the design map) match central finite differences of the
same responses within 1e-6 relative (volume) and 1e-5 relative (compliance,
whose differences carry the direct solve's rounding); the displacement at a
parametric point and its three-adjoint gradient match differences within
1e-6 (step 1e-4); an SLSQP loop
(scipy) over four thickness variables of the cantilever lowers its
compliance at fixed volume.  The host logic (listpatch validation, the
propagation through a coarse-to-fine map, the finite-difference helper, the
rational basis at a parametric point) runs on the CPU.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import load_fixture
from yeti_b200.optimization import ShapeOptimization
from yeti_b200.stiffmtrx_elemstorage import SYSTEM_ARG_NAMES


def cantilever_problem(**kw):
    """10x1x1 cantilever (p=2, 16x4x4), clamped at x=0, tip traction -z on
    x=10.  Variable v (0..3) lifts the top-face control points of the slab
    2.5 v <= x < 2.5 (v+1) by x_v; the loaded tip face does not move."""
    _, args = load_fixture("cantilever_p2_16x4x4")
    X = np.asarray(dict(zip(SYSTEM_ARG_NAMES, args))["COORDS3D"], dtype=np.float64)
    top = np.abs(X[2] - 1.0) < 1e-12
    tip = np.abs(X[0] - 10.0) < 1e-12
    slab = np.minimum((X[0] / 2.5).astype(int), 3)
    masks = [top & ~tip & (slab == v) for v in range(4)]

    def update(c0, x):
        c = c0.copy()
        for v in range(4):
            c[2, masks[v]] += x[v]
        return c

    def d_update(c0, x, ivar):
        d = np.zeros_like(c0)
        d[2, masks[ivar]] = 1.0
        return d

    return ShapeOptimization(args, 4, update, d_update_function=d_update, **kw), args


# ---------------------------------------------------------------------- CPU
def test_listpatch_and_shape_validation():
    opt, _ = cantilever_problem()
    x = np.zeros(4)
    with pytest.raises(ValueError, match="Length of listpatch"):
        opt.volume(x, listpatch=np.array([1, 1]))
    with pytest.raises(ValueError, match="0 or 1"):
        opt.volume(x, listpatch=np.array([2]))
    with pytest.raises(ValueError, match="expected 4"):
        opt.compliance(np.zeros(3))
    bad = ShapeOptimization(opt.args, 1, lambda c0, x: c0[:, :5])
    with pytest.raises(ValueError, match="update_function returned shape"):
        bad.design_coords(np.zeros(1))
    with pytest.raises(ValueError, match="coarse_to_fine has shape"):
        ShapeOptimization(opt.args, 1, lambda c0, x: c0, coarse_to_fine=sp.eye(5))


def test_propagation_through_map_and_fd_fallback():
    """The propagated gradient equals sum_ij dP_design/dx (M^T g)_ij, with the
    derivative given or taken by central differences of the update."""
    _, args = load_fixture("quarter_annulus_p2_4x4x2")
    X0 = np.asarray(dict(zip(SYSTEM_ARG_NAMES, args))["COORDS3D"], dtype=np.float64)
    n = X0.shape[1]
    rng = np.random.default_rng(3)
    S = sp.random(n, n, density=0.05, random_state=4, format="csr")
    M = sp.eye(n, format="csr") + 0.01 * S
    D = rng.standard_normal((3, 3, n))        # coords = c0 + sum_v x_v D_v

    def update(c0, x):
        return c0 + np.tensordot(x, D, axes=1) + 0.1 * x[0] ** 2 * D[1]

    def d_update(c0, x, ivar):
        return D[ivar] + (0.2 * x[0] * D[1] if ivar == 0 else 0.0)

    g_fine = rng.standard_normal((3, n))
    x = np.array([0.3, -0.2, 0.1])
    g_design = (M.T @ g_fine.T).T
    want = np.array([np.sum(d_update(X0, x, i) * g_design) for i in range(3)])
    a = ShapeOptimization(args, 3, update, coarse_to_fine=M, d_update_function=d_update)
    b = ShapeOptimization(args, 3, update, coarse_to_fine=M)
    np.testing.assert_allclose(a.propagate(x, g_fine), want, rtol=1e-13)
    np.testing.assert_allclose(b.propagate(x, g_fine), want, rtol=1e-8)
    np.testing.assert_allclose(a.analysis_coords(x), (M @ update(X0, x).T).T, rtol=1e-15)


def test_finite_difference_helper():
    opt, _ = cantilever_problem()
    f = lambda x: x[0] ** 3 + 2.0 * x[1] * x[2] - x[3]
    x = np.array([1.0, 2.0, 3.0, 4.0])
    exact = np.array([3.0, 6.0, 4.0, -1.0])
    np.testing.assert_allclose(opt._sensitivity_fd(f, x, 1e-6, True), exact, rtol=1e-8)
    np.testing.assert_allclose(opt._sensitivity_fd(f, x, 1e-7, False), exact, rtol=1e-5)


def test_point_basis_geometry():
    """The rational basis at a parametric point: it sums to 1, interpolates
    the corner control point, reproduces the cantilever's affine map
    x = (10 xi, eta, zeta) (linear precision of B-splines) and keeps the
    quarter annulus's exact arcs (in-plane radius constant along eta)."""
    opt, args = cantilever_problem()
    X = np.asarray(dict(zip(SYSTEM_ARG_NAMES, args))["COORDS3D"], dtype=np.float64)
    rng = np.random.default_rng(7)
    for xi in list(rng.random((20, 3))) + [np.array([0.0, 0.0, 0.0]), np.array([1.0, 1.0, 1.0]),
                                          np.array([0.5, 0.25, 0.75])]:
        cps, R = opt.point_basis(xi)
        assert abs(R.sum() - 1.0) < 1e-14
        x = R @ X[:, cps].T
        np.testing.assert_allclose(x, [10 * xi[0], xi[1], xi[2]], atol=1e-13)
    cps, R = opt.point_basis([0.0, 0.0, 0.0])
    corner = np.argmin(np.abs(X - X.min(axis=1, keepdims=True)).sum(axis=0))
    assert R.max() == pytest.approx(1.0, abs=1e-15) and cps[np.argmax(R)] == corner
    with pytest.raises(ValueError, match="outside"):
        opt.point_basis([1.2, 0.5, 0.5])
    _, a2 = load_fixture("quarter_annulus_p2_4x4x2")
    Xa = np.asarray(dict(zip(SYSTEM_ARG_NAMES, a2))["COORDS3D"], dtype=np.float64)
    ann = ShapeOptimization(a2, 1, lambda c0, x: c0)
    for u in (0.0, 0.3, 0.77, 1.0):
        radii = []
        for v in np.linspace(0.0, 1.0, 9):
            cps, R = ann.point_basis([u, v, 0.4])
            x = R @ Xa[:, cps].T
            radii.append(np.hypot(x[0], x[1]))
        assert np.ptp(radii) < 1e-12 * max(radii)


def test_displacement_fd_shape():
    """Vector responses give (nb_var, m) differences."""
    opt, _ = cantilever_problem()
    g = opt._sensitivity_fd(lambda y: np.array([y[0] ** 2, y[1] * y[2], y[3]]),
                            np.array([1.0, 2.0, 3.0, 4.0]), 1e-6, True)
    np.testing.assert_allclose(g, [[2, 0, 0], [0, 3, 0], [0, 2, 0], [0, 0, 1]], atol=1e-8)


# ---------------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_responses_equal_moved_model(cuda_ok):
    from yeti_b200.gradient import _solve
    from yeti_b200.volume import computevolume
    opt, args = cantilever_problem()
    x = np.array([0.05, -0.02, 0.03, 0.01])
    X = opt.analysis_coords(x)
    U, F = _solve(args, X)
    assert opt.compliance(x) == 0.5 * float(U @ F)
    d = dict(zip(SYSTEM_ARG_NAMES, args))
    A = [np.ones(1, dtype=np.int64), X, d["IEN"], d["nb_elem_patch"], d["Nkv"], d["Ukv"],
         d["Nijk"], d["weight"], d["Jpqr"], d["ELT_TYPE"], d["PROPS"], d["JPROPS"],
         d["TENSOR"], d["MCRD"], d["NBINT"], d["NNODE"]]
    assert opt.volume(x) == computevolume(*A)
    # only z coordinates move, so det J and the volume are linear in x
    x0 = np.zeros(4)
    lin = opt.volume(x0) + opt.grad_volume_analytic(x0) @ x
    assert abs(opt.volume(x) - lin) <= 1e-12 * opt.volume(x0)
    assert abs(opt.volume(x0) - 10.0) <= 1e-12 * 10.0


@pytest.mark.gpu
def test_analytic_gradients_vs_finite_differences(cuda_ok):
    opt, _ = cantilever_problem()
    x = np.array([0.05, -0.02, 0.03, 0.01])
    gv = opt.grad_volume_analytic(x)
    fv = opt.grad_volume_finite_differences(x, eps=1e-6, centered=True)
    assert np.linalg.norm(gv - fv) <= 1e-6 * np.linalg.norm(fv)
    gc = opt.grad_compliance_analytic(x)
    fc = opt.grad_compliance_finite_differences(x, eps=1e-6, centered=True)
    assert np.linalg.norm(gc - fc) <= 1e-5 * np.linalg.norm(fc)
    # thicker near the clamp lowers the compliance most
    assert gc[0] < gc[1] < gc[2] < gc[3] < 0


@pytest.mark.gpu
def test_displacement_and_its_analytic_gradient(cuda_ok):
    """u(xi) = sum R_a(xi) U_a of the GPU solution, and du/dx from three
    adjoint solves and the GPU adjoint kernel (three adjoints in one call)
    against central differences.  The step is 1e-4: the differences of this
    slender, stiff model carry the direct solve's rounding divided by the
    step (2e-6 relative at 1e-6, 3e-8 at 1e-4 with the CPU oracle)."""
    from yeti_b200.gradient import _solve
    opt, args = cantilever_problem()
    x = np.array([0.05, -0.02, 0.03, 0.01])
    for xi in ([1.0, 0.5, 1.0], [0.6, 0.3, 0.8]):
        U = _solve(args, opt.analysis_coords(x))[0]
        cps, R = opt.point_basis(xi)
        u = opt.displacement(x, xi)
        np.testing.assert_array_equal(u, R @ U.reshape(-1, 3)[cps])
        ga = opt.grad_displacement_analytic(x, xi)
        gf = opt.grad_displacement_finite_differences(x, xi, eps=1e-4, centered=True)
        assert ga.shape == gf.shape == (4, 3)
        assert np.linalg.norm(ga - gf) <= 1e-6 * np.linalg.norm(gf)
    # the tip deflects downwards under the -z traction; lifting the top face
    # near the clamp stiffens the beam: d u_z / d x_0 > 0
    assert opt.displacement(x, [1.0, 0.5, 0.5])[2] < 0
    assert opt.grad_displacement_analytic(x, [1.0, 0.5, 0.5])[0, 2] > 0


@pytest.mark.gpu
def test_gradients_through_coarse_to_fine_map(cuda_ok):
    """The same responses with a design model mapped to the analysis model by
    a fixed sparse linear map (translations preserved): AN vs central FD."""
    _, args = load_fixture("quarter_annulus_p2_4x4x2")
    X0 = np.asarray(dict(zip(SYSTEM_ARG_NAMES, args))["COORDS3D"], dtype=np.float64)
    n = X0.shape[1]
    S = sp.random(n, n, density=0.03, random_state=5, format="csr")
    S = S - sp.diags(np.asarray(S.sum(axis=1)).ravel())
    M = sp.eye(n, format="csr") + 0.005 * S
    thick = np.abs(X0[2] - X0[2].max()) < 1e-12

    def update(c0, x):
        c = c0.copy()
        c[2, thick] += x[0]
        c[0] *= 1.0 + x[1]
        return c

    # both variables move the pressure-loaded outer face: the analytic
    # gradient needs the surface-load term to match the differences
    opt = ShapeOptimization(args, 2, update, coords_0=X0, coarse_to_fine=M,
                            include_surface_loads=True)
    x = np.array([0.01, 0.02])
    gv = opt.grad_volume_analytic(x)
    fv = opt.grad_volume_finite_differences(x, eps=1e-6, centered=True)
    assert np.linalg.norm(gv - fv) <= 1e-6 * np.linalg.norm(fv)
    gc = opt.grad_compliance_analytic(x)
    fc = opt.grad_compliance_finite_differences(x, eps=1e-6, centered=True)
    assert np.linalg.norm(gc - fc) <= 1e-5 * np.linalg.norm(fc)


@pytest.mark.gpu
def test_slsqp_lowers_compliance_at_fixed_volume(cuda_ok):
    from scipy.optimize import minimize
    opt, _ = cantilever_problem()
    x0 = np.zeros(4)
    c0, v0 = opt.compliance(x0), opt.volume(x0)
    res = minimize(opt.compliance, x0, jac=opt.grad_compliance_analytic, method="SLSQP",
                   bounds=[(-0.3, 0.3)] * 4,
                   constraints=[{"type": "ineq", "fun": lambda x: v0 - opt.volume(x),
                                 "jac": lambda x: -opt.grad_volume_analytic(x)}],
                   options={"maxiter": 8})
    assert opt.compliance(res.x) < 0.95 * c0
    assert opt.volume(res.x) <= v0 * (1 + 1e-6)
    assert res.x[0] > 0 > res.x[3]
