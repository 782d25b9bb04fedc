"""Generate golden weighted-quadrature OPERATOR products from the reference's
own Python WQ assembly.

The reference ships a pure-Python twin of its WQ assembly,
``iga_wq_mf/ThermoMechaIGA/pysrc/lib/methods_wq.py`` (class ``WQ``):

* ``eval_basis_weights`` (``methods_wq.py:40-66``) builds the 1-D B0, B1,
  W00, W01, W10, W11 of every direction with ``wq_find_basis_weights_opt``
  (``base_functions.py:565-670``);
* ``eval_jacobien_pps`` (``create_model.py:531-568``) gives the B-spline
  Jacobian ``J[i, j, q] = dx_i / dxi_j`` at the WQ points;
* ``eval_K_C_coefficient`` (``create_model.py:570-601``) gives the scalar
  conductivity coefficient ``inv(J) inv(J)^T det(J)``;
* ``eval_conductivity_matrix`` (``methods_wq.py:76-108``) assembles
  ``K = sum_{i,j} (W^{(i,j)} diag(C_ij)) B^{(j)T}`` with Kronecker products of
  the 1-D matrices (test derivative i, trial derivative j).

The elastic operator is the 3 x 3 block matrix whose block (a, b) is that
same assembly with ``C_kl = S[(a,k), (b,l)]`` (``wq_get_stiffness_3d``,
``wq_assembly.f90:1020-1054``), S being the Fortran's elastic coefficient
``ext(invJ)^T MDM ext(invJ) detJ`` (``eval_mech_coefficient``,
``wq_assembly.f90:52-138``; restated below, the only step the reference has
in Fortran alone).  That Fortran product uses the transpose of the
geometric inverse; it agrees with the geometric form wherever the Jacobian
is symmetric, so the elastic cases use geometries with symmetric Jacobians:
an axis-aligned box and maps x = grad(phi) of a cubic potential (Jacobian =
Hessian of phi).  General (perturbed) patches pin the Jacobian, the
conductivity coefficient and the scalar operator instead.

All cases have unit weights (the reference's WQ geometry is a B-spline).
The reference's modules import packages that are absent here (matplotlib,
pyevtk, geomdl, the f2py module ``iga_wq_mf``, YETI's preprocessing): they are
stubbed; ``geomdl.helpers`` is restated (see make_wq_golden.py).

Writes tests/golden/wq_operator.npz.
Usage:  YETI_REFERENCE=<reference root> python tests/golden/make_wq_operator_golden.py
"""
import importlib
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import make_wq_golden  # noqa: E402

E, NU = 1.0, 0.3

# (name, p, nel, geometry); "box": axis-aligned box (1.3, 0.7, 2.1),
# "sym": x = grad(phi), "gen": perturbed control points
CASES = [
    ("box_p4", 4, (2, 3, 2), "box"),
    ("sym_p2", 2, (3, 2, 4), "sym"),
    ("sym_p3", 3, (2, 3, 2), "sym"),
    ("sym_p2_long", 2, (7, 2, 3), "sym"),     # n = 9 > p + 3: copied interior rows
    ("gen_p2", 2, (2, 4, 3), "gen"),
    ("gen_p3", 3, (3, 2, 2), "gen"),
]


def load_reference_wq():
    """Import methods_wq.WQ from the reference tree with its absent
    dependencies stubbed."""
    bf = make_wq_golden.load_base_functions()   # installs geomdl.helpers

    def stub(name, **attrs):
        m = sys.modules.get(name) or types.ModuleType(name)
        for k, v in attrs.items():
            setattr(m, k, v)
        sys.modules[name] = m
        return m

    class IGAparametrization:   # isinstance checks only
        pass

    stub("preprocessing")
    stub("preprocessing.igaparametrization", IGAparametrization=IGAparametrization)
    stub("matplotlib")
    stub("matplotlib.pyplot")
    stub("pyevtk")
    stub("pyevtk.hl", gridToVTK=None)
    stub("iga_wq_mf.assembly")
    sys.modules["iga_wq_mf"].assembly = sys.modules["iga_wq_mf.assembly"]
    g = stub("geomdl", fitting=None, BSpline=None, operations=None)
    g.helpers = sys.modules["geomdl.helpers"]
    pkg = types.ModuleType("refwq")
    pkg.__path__ = [os.path.join(make_wq_golden.reference_root(), make_wq_golden.LIB)]
    sys.modules["refwq"] = pkg
    mw = importlib.import_module("refwq.methods_wq")
    return mw.WQ, bf


def collocation(bf, p, kv, x):
    """N_j(x_i): B-spline values of the uniform open knot vector kv."""
    n = len(kv) - p - 1
    C = np.zeros((len(x), n))
    for i, t in enumerate(x):
        span = make_wq_golden.find_span_linear(p, kv, n, t)
        d = make_wq_golden.basis_function_ders(p, kv, span, t, 0)
        C[i, span - p:span + 1] = d[0]
    return C


def interpolate_map(bf, p, nel, fmap):
    """Control points (ncp, 3) of the spline interpolant of fmap at the
    Greville abscissae (exact for maps in the spline space)."""
    kvs, gs, Cs = [], [], []
    for d in range(3):
        kv = np.asarray(bf.create_knotvector(p, nel[d]), dtype=np.float64)
        n = p + nel[d]
        g = np.array([kv[i + 1:i + p + 1].mean() for i in range(n)])
        kvs.append(kv)
        gs.append(g)
        Cs.append(collocation(bf, p, kv, g))
    W, V, U = np.meshgrid(gs[2], gs[1], gs[0], indexing="ij")
    vals = fmap(U, V, W)                       # (3, nw, nv, nu)
    inv = [np.linalg.inv(C) for C in Cs]
    cp = np.einsum("cwvu,au,bv,dw->cdba", vals, inv[0], inv[1], inv[2])
    return cp.reshape(3, -1).T.copy()          # u fastest


def geometry(kind, p, nel, rng, bf):
    if kind == "box":
        s = np.array([1.3, 0.7, 2.1])
        return interpolate_map(bf, p, nel, lambda u, v, w: np.stack([s[0] * u, s[1] * v, s[2] * w]))
    if kind == "sym":
        s, eps = (1.3, 0.8, 1.1), 0.15

        # phi = sum s_d xi_d^2 / 2 + eps (u^2 v + v^2 w + w^2 u + u v w)
        def grad_phi(u, v, w):
            return np.stack([s[0] * u + eps * (2 * u * v + w * w + v * w),
                             s[1] * v + eps * (u * u + 2 * v * w + u * w),
                             s[2] * w + eps * (v * v + 2 * w * u + u * v)])
        return interpolate_map(bf, p, nel, grad_phi)
    # perturbed unit-cube patch, boundary CPs on the faces
    cp = interpolate_map(bf, p, nel, lambda u, v, w: np.stack([u, v, w]))
    n = [p + nel[d] for d in range(3)]
    iw, iv, iu = np.meshgrid(np.arange(n[2]), np.arange(n[1]), np.arange(n[0]), indexing="ij")
    inner = ((iu > 0) & (iu < n[0] - 1) & (iv > 0) & (iv < n[1] - 1) &
             (iw > 0) & (iw < n[2] - 1)).ravel()
    for d in range(3):
        h = 1.0 / nel[d]
        cp[:, d] += np.where(inner, rng.uniform(-0.2 * h, 0.2 * h, cp.shape[0]), 0.0)
    return cp


def mech_coefficient(J):
    """eval_mech_coefficient (wq_assembly.f90:52-138):
    S = ext(invJ)^T (MM^T DD MM) ext(invJ) detJ per point, DD the isotropic
    elasticity (material_lib.f90:75-87)."""
    lam = E * NU / ((1 + NU) * (1 - 2 * NU))
    mu = E / (2 * (1 + NU))
    DD = np.zeros((6, 6))
    DD[:3, :3] = lam
    DD[range(3), range(3)] = lam + 2 * mu
    DD[3, 3] = DD[4, 4] = DD[5, 5] = mu
    MM = np.zeros((6, 9))
    for r, c in ((1, 1), (2, 5), (3, 9), (4, 2), (4, 4), (5, 6), (5, 8), (6, 3), (6, 7)):
        MM[r - 1, c - 1] = 1.0
    MDM = MM.T @ DD @ MM
    nq = J.shape[2]
    S = np.empty((9, 9, nq))
    for q in range(nq):
        invJ = np.linalg.inv(J[:, :, q])
        X = np.zeros((9, 9))
        for k in range(3):
            X[3 * k:3 * k + 3, 3 * k:3 * k + 3] = invJ
        S[:, :, q] = X.T @ MDM @ X * np.linalg.det(J[:, :, q])
    return S


def main():
    WQ, bf = load_reference_wq()
    rng = np.random.default_rng(20261203)
    out = {}
    for name, p, nel, kind in CASES:
        cps = geometry(kind, p, nel, rng, bf)
        ncp = cps.shape[0]
        wq = WQ.__new__(WQ)                    # the model-file constructor is not used
        wq._dim = 3
        wq._degree = np.array([[p], [p], [p]])
        wq._knotvector = [[np.asarray(bf.create_knotvector(p, nel[d]), dtype=np.float64)
                           for d in range(3)]]
        wq._r_ = 2
        wq._nb_ctrlpts_total = ncp
        wq.eval_basis_weights()
        nqp = int(np.prod([wq._DB[d][0].shape[1] for d in range(3)]))
        J, _ = wq.eval_jacobien_pps(3, cps, wq._DB, nqp)
        out[f"{name}_p"] = np.array([p, p, p])
        out[f"{name}_nel"] = np.array(nel)
        out[f"{name}_cps"] = cps.T.copy()      # (3, ncp)
        out[f"{name}_J"] = J
        if kind == "gen":
            Kc, _, detJ = wq.eval_K_C_coefficient(nqp, J, np.eye(3), 1.0)
            wq._conductivity_coef = Kc
            K = wq.eval_conductivity_matrix().tocsr()
            X = rng.standard_normal((ncp, 3))
            out[f"{name}_kcoef"] = Kc
            out[f"{name}_X"] = X
            out[f"{name}_KX"] = K @ X
        else:
            assert np.abs(J - np.swapaxes(J, 0, 1)).max() < 1e-12 * np.abs(J).max()
            assert np.linalg.det(np.moveaxis(J, 2, 0)).min() > 0
            S = mech_coefficient(J)
            X = rng.standard_normal((3 * ncp, 3))
            KX = np.zeros_like(X)
            for a in range(3):
                for b in range(3):
                    wq._conductivity_coef = S[3 * a:3 * a + 3, 3 * b:3 * b + 3, :]
                    Kab = wq.eval_conductivity_matrix().tocsr()
                    KX[a * ncp:(a + 1) * ncp] += Kab @ X[b * ncp:(b + 1) * ncp]
            out[f"{name}_X"] = X
            out[f"{name}_KX"] = KX
        print(name, "ncp", ncp, "nqp", nqp)
    np.savez_compressed(os.path.join(HERE, "wq_operator.npz"), **out)


if __name__ == "__main__":
    main()
