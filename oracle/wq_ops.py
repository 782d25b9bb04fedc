"""FP64 numpy oracle of the weighted-quadrature (WQ) elastic operator on a
single NURBS patch.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Pinned to the reference's own Python WQ assembly (methods_wq.WQ,
iga_wq_mf/ThermoMechaIGA/pysrc/lib/methods_wq.py:76-108, with its
eval_jacobien_pps / eval_K_C_coefficient, create_model.py:531-601) by
tests/golden/wq_operator.npz (generator: tests/golden/make_wq_operator_golden.py):
the elastic operator, assembled there block by block from the Fortran's
coefficient formula, on geometries with symmetric Jacobians (where the
Fortran's orientation and the geometric one agree); the Jacobian, the
conductivity coefficient and the scalar operator on perturbed patches.  The
1-D rules are pinned to the reference's Python twin (tests/golden/
wq_rules.npz); tests/test_wq.py adds exactness on affine patches, a dense
direct solve and the reference's rank-one algorithm (oracle/oracle_wq.c).

The reference ships the WQ matrix-free operator for the scalar (thermal)
problem only, with B-spline geometry:
  * K u = sum_{k,l} W^{(k,l)} (coef_kl * (B^{(l)})^T u)
    (mf_wq_get_ku_3d, src/yeti_iga/iga_wq_mf/fsrc/mf_wq_solver.f90:284-544),
    W^{(k,l)} the Kronecker product of the 1-D weights W^{[d==k][d==l]} and
    B^{(l)} that of B^{[d==l]};
  * the elastic coefficient S = ext(invJ)^T (MM^T DD MM) ext(invJ) detJ
    (eval_mech_coefficient, wq_assembly.f90:52-138), used per 3x3 component
    block (wq_get_stiffness_3d, wq_assembly.f90:1020-1054);
  * the Jacobian from B-spline sums (jacobien_physicalposition_3d,
    wq_assembly.f90:233-473).
This oracle composes them into the elastic operator

    (K U)_{a,i} = sum_{k,l} sum_q W^{(k,l)}_a(q) sum_j S[(i,k),(j,l)](q) (B^{(l)} U_j)(q)

with the reference's B-spline test and trial functions, on the exact NURBS
geometry: the Jacobian J = dx/dxi of x = sum w_a N_a P_a / sum w_a N_a.

Two deliberate differences from the reference's code: the coefficient uses
the geometric orientation
S = ext(invJ) MDM ext(invJ)^T |detJ| with invJ = (dx/dxi)^{-1} (the
reference's product is transposed, which only agrees for symmetric
Jacobians), and the Jacobian includes the NURBS weights.  Rational
(NURBS) test and trial functions were tried and rejected: under weighted
quadrature their value/derivative coupling terms make the operator lose
coercivity on the randomly weighted patches of the benchmark (CG and BiCGSTAB
fail from 32^3 elements up), while the B-spline space stays solvable.
"""
import numpy as np

from . import wq_rules


def material_threed(E, nu):
    """ddsdde of material_lib.f90:75-87 (Voigt 11,22,33,12,13,23)."""
    lam = (E * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] = lam + 2.0 * mu
    D[3, 3] = D[4, 4] = D[5, 5] = mu
    return D


def mdm_matrix(E, nu):
    """MM^T DD MM (wq_assembly.f90:92-109): the 9x9 elasticity in terms of
    the displacement gradient g[(c)*3 + d] = du_c/dx_d."""
    MM = np.zeros((6, 9))
    for r, c in ((0, 0), (1, 4), (2, 8), (3, 1), (3, 3), (4, 5), (4, 7),
                 (5, 2), (5, 6)):
        MM[r, c] = 1.0
    return MM.T @ material_threed(E, nu) @ MM


def _fwd(f, Bu, Bv, Bw):
    """(nw, nv, nu) field on functions -> (qw, qv, qu) values at points:
    t[w,v,q] = sum_u f[w,v,u] Bu[u,q], then along v, then along w (matrix
    products, so that the full-size operators run through BLAS)."""
    t = f @ Bu                                   # (w, v, q)
    t = np.matmul(Bv.T, t)                       # (w, r, q)
    nw, nr, nq = t.shape
    return (Bw.T @ t.reshape(nw, nr * nq)).reshape(-1, nr, nq)


def _bwd(h, Wu, Wv, Ww):
    """(qw, qv, qu) point values -> (nw, nv, nu) with the 1-D weights."""
    t = h @ Wu.T                                 # (s, r, u)
    t = np.matmul(Wv, t)                         # (s, v, u)
    ns, nv, nu = t.shape
    return (Ww @ t.reshape(ns, nv * nu)).reshape(-1, nv, nu)


class WQOracle:
    """FP64 WQ elasticity on one patch (see module docstring)."""

    def __init__(self, patch, E, nu, clamp_faces=None):
        from yeti_b200.patches import free_mask
        self.p = tuple(patch["p"])
        self.nel = tuple(patch["nel"])
        self.n = [self.p[d] + self.nel[d] for d in range(3)]
        self.rules = [wq_rules.wq_rule(self.p[d], self.nel[d]) for d in range(3)]
        nu_, nv_, nw_ = self.n
        self.w = patch["weights"].reshape(nw_, nv_, nu_)   # geometry weights
        X = patch["cps"].reshape(3, nw_, nv_, nu_)
        self.mask = free_mask(patch, clamp_faces).reshape(3, nw_, nv_, nu_)
        self.ndof = 3 * nu_ * nv_ * nw_
        self._geometry(X, E, nu)

    def _B(self, d, order):
        return self.rules[d]["B1" if order else "B0"]

    def _W(self, d, test, trial):
        return self.rules[d][f"W{int(test)}{int(trial)}"]

    def fwd(self, f, lam):
        """Trial kind lam (0 value, 1..3 derivative direction) at points."""
        return _fwd(f, self._B(0, lam == 1), self._B(1, lam == 2),
                    self._B(2, lam == 3))

    def bwd(self, h, kappa, lam):
        return _bwd(h, self._W(0, kappa == 1, lam == 1),
                    self._W(1, kappa == 2, lam == 2),
                    self._W(2, kappa == 3, lam == 3))

    def _geometry(self, X, E, nu):
        w = self.w
        Xw = [w * X[0], w * X[1], w * X[2], w]
        V = [self.fwd(f, 0) for f in Xw]
        D = [[self.fwd(f, l) for l in (1, 2, 3)] for f in Xw]
        W = V[3]
        gW = np.stack(D[3])                       # (3, qw, qv, qu)
        x = np.stack(V[:3]) / W
        J = np.empty((3, 3) + W.shape)
        for c in range(3):
            for l in range(3):
                J[c, l] = (D[c][l] - x[c] * gW[l]) / W
        Jq = np.moveaxis(J, (0, 1), (-2, -1))     # (..., 3, 3)
        self.J = J                                # J[c, l] = dx_c / dxi_l
        self.detJ = np.linalg.det(Jq)
        invJ = np.linalg.inv(Jq)                  # invJ[..., k, d] = dxi_k/dx_d
        MDM = mdm_matrix(E, nu)
        P = np.zeros(Jq.shape[:-2] + (9, 9))
        for c in range(3):
            P[..., 3 * c:3 * c + 3, 3 * c:3 * c + 3] = invJ
        self.S = P @ MDM @ np.swapaxes(P, -1, -2) * np.abs(self.detJ)[..., None, None]
        self.W = W
        self.x = x

    # ------------------------------------------------------------ operator
    def apply(self, u):
        u = np.asarray(u, dtype=np.float64).reshape(self.mask.shape) * self.mask
        F = [[self.fwd(u[j], l) for j in range(3)] for l in (1, 2, 3)]
        S = self.S
        out = np.zeros_like(u)
        for i in range(3):
            acc = 0.0
            for k in (1, 2, 3):
                for l in (1, 2, 3):
                    h = sum(S[..., 3 * i + k - 1, 3 * j + l - 1] * F[l - 1][j]
                            for j in range(3))
                    acc = acc + self.bwd(h, k, l)
            out[i] = acc
        return (out * self.mask).ravel()

    def conductivity_coef(self):
        """Scalar conductivity coefficient inv(J) inv(J)^T |det J| per point,
        (3, 3, nqp) with the points u fastest (eval_K_C_coefficient,
        create_model.py:570-601, with an identity conductivity)."""
        Jq = np.moveaxis(self.J, (0, 1), (-2, -1))
        invJ = np.linalg.inv(Jq)
        C = invJ @ np.swapaxes(invJ, -1, -2) * np.abs(self.detJ)[..., None, None]
        return np.moveaxis(C, (-2, -1), (0, 1)).reshape(3, 3, -1)

    def apply_scalar(self, u, coef):
        """Scalar WQ operator sum_{k,l} W^{(k,l)} (coef_kl * (B^{(l)})^T u)
        on one field of control-point values (mf_wq_get_ku_3d,
        mf_wq_solver.f90:284-544; no clamps).  coef: (3, 3, nqp), points u
        fastest."""
        shp = self.mask.shape[1:]
        u = np.asarray(u, dtype=np.float64).reshape(shp)
        C = np.asarray(coef).reshape((3, 3) + self.detJ.shape)
        G = [self.fwd(u, l) for l in (1, 2, 3)]
        out = np.zeros(shp)
        for k in (1, 2, 3):
            for l in (1, 2, 3):
                out += self.bwd(C[k - 1, l - 1] * G[l - 1], k, l)
        return out.ravel()

    def diag(self):
        S = self.S
        out = np.zeros(self.mask.shape)
        for i in range(3):
            acc = 0.0
            for k in (1, 2, 3):
                for l in (1, 2, 3):
                    mats = [self._W(d, k == d + 1, l == d + 1) *
                            self._B(d, l == d + 1) for d in range(3)]
                    acc = acc + _bwd(S[..., 3 * i + k - 1, 3 * i + l - 1], *mats)
            out[i] = acc
        out = np.where(self.mask > 0, out, 1.0)
        return out.ravel()

    def body_force(self, f):
        """Load vector of a constant force density f (wq_get_force_3d,
        wq_assembly.f90:1193-1251)."""
        out = np.zeros(self.mask.shape)
        for i in range(3):
            out[i] = self.bwd(f[i] * np.abs(self.detJ), 0, 0)
        return (out * self.mask).ravel()

    def matrix(self):
        """Explicit operator (small patches only)."""
        n = self.ndof
        K = np.zeros((n, n))
        e = np.zeros(n)
        for c in range(n):
            e[c] = 1.0
            K[:, c] = self.apply(e)
            e[c] = 0.0
        return K

    # ------------------------------------------ fast diagonalisation
    def fd_box(self, c):
        """Free function range [lo, hi) along u, v, w of component c."""
        m = self.mask[c] > 0                       # (nw, nv, nu)
        out = []
        for axes in ((0, 1), (0, 2), (1, 2)):      # reduce to u, v, w
            idx = np.nonzero(m.any(axis=axes))[0]
            out.append((int(idx[0]), int(idx[-1]) + 1))
        return out

    def fd_1d(self, d, lo, hi):
        """Restricted, symmetrised 1-D WQ matrices (K, M) = (W11 B1^T,
        W00 B0^T) of direction d (eigen_decomposition's KK and MM,
        tensor_algebra.f90:1038-1063)."""
        R = self.rules[d]
        M = (R["W00"] @ R["B0"].T)[lo:hi, lo:hi]
        K = (R["W11"] @ R["B1"].T)[lo:hi, lo:hi]
        return 0.5 * (K + K.T), 0.5 * (M + M.T)

    def td_weights(self, c, sweeps=2):
        """Per-point 1-D weights (M, K) of component c from `sweeps` sweeps
        of tensor_decomposition_3d (tensor_algebra.f90:1256-1382) over its
        diagonal coefficients S[(c,k),(c,k)]; the direction-3 slices run
        over the w points (the reference bounds that loop by the v count,
        the same whenever the two agree)."""
        CC = [self.S[..., 3 * c + k, 3 * c + k] for k in range(3)]   # (qw, qv, qu)
        nq = [CC[0].shape[2], CC[0].shape[1], CC[0].shape[0]]
        M = [np.ones(nq[d]) for d in range(3)]
        K = [np.ones(nq[d]) for d in range(3)]
        axis = {0: 2, 1: 1, 2: 0}                 # grid axis of direction d
        others = {d: tuple(a for a in range(3) if a != axis[d]) for d in range(3)}

        def grid(v, d):
            shape = [1, 1, 1]
            shape[axis[d]] = v.size
            return v.reshape(shape)
        for _ in range(sweeps):
            for k in range(3):
                uu = [grid(M[d], d) for d in range(3)]
                V = CC[k] * uu[k] / (uu[0] * uu[1] * uu[2])
                K[k] = np.sqrt(V.min(axis=others[k]) * V.max(axis=others[k]))
            for k in range(3):
                uu = [grid(M[d], d) for d in range(3)]
                ww = grid(K[k], k)
                W = [CC[k] * uu[k] * uu[l] / (uu[0] * uu[1] * uu[2] * ww)
                     for l in range(3) if l != k]
                N = np.minimum(W[0], W[1])
                X = np.maximum(W[0], W[1])
                M[k] = np.sqrt(N.min(axis=others[k]) * X.max(axis=others[k]))
        return M, K

    def fd_1d_weighted(self, d, lo, hi, mw, kw):
        """1-D matrices of the 'TD' branch of eigen_decomposition
        (tensor_algebra.f90:1045-1071): W00 (B0 diag(mw))^T and W11 (B1
        diag(kw))^T restricted, symmetrised by averaging with the transpose
        (the reference hands the non-symmetric products to dsygvd, which
        reads the upper triangle; that triangle is indefinite on rough
        coefficient fields)."""
        R = self.rules[d]
        M = (R["W00"] @ (R["B0"] * mw[None, :]).T)[lo:hi, lo:hi]
        K = (R["W11"] @ (R["B1"] * kw[None, :]).T)[lo:hi, lo:hi]
        return 0.5 * (K + K.T), 0.5 * (M + M.T)

    def fd_setup(self, scaled=False, unit=False, td=False):
        """Per component: box, eigenpairs of K_d U = M_d U lam (scipy's
        generalised symmetric solver, U^T M U = I), coefficients a[c][d]
        (1, or the mean over the points of S[(c,d),(c,d)]) and, when scaled,
        s = sqrt(diag(P) / diag(K)) (find_parametric_diag_3d and
        scaling_FastDiag, tensor_algebra.f90:1452-1482, 1598-1625)."""
        from scipy.linalg import eigh
        dK = self.diag().reshape(self.mask.shape)
        plan = []
        for c in range(3):
            box = self.fd_box(c)
            a = [1.0 if (unit or td) else float(self.S[..., 3 * c + d, 3 * c + d].mean())
                 for d in range(3)]
            eig, dg = [], []
            if td:
                tM, tK = self.td_weights(c)
            for d, (lo, hi) in enumerate(box):
                if td:
                    K, M = self.fd_1d_weighted(d, lo, hi, tM[d], tK[d])
                else:
                    K, M = self.fd_1d(d, lo, hi)
                lam, U = eigh(K, M)
                eig.append((lam, U))
                dg.append((np.diag(K).copy(), np.diag(M).copy()))
            lam3 = (a[2] * eig[2][0][:, None, None] + a[1] * eig[1][0][None, :, None]
                    + a[0] * eig[0][0][None, None, :])
            s = None
            if scaled:
                (ku, mu), (kv, mv), (kw, mw) = dg
                dp = (a[0] * mw[:, None, None] * mv[None, :, None] * ku[None, None, :]
                      + a[1] * mw[:, None, None] * kv[None, :, None] * mu[None, None, :]
                      + a[2] * kw[:, None, None] * mv[None, :, None] * mu[None, None, :])
                sl = tuple(slice(*box[d]) for d in (2, 1, 0))
                s = np.sqrt(dp / dK[c][sl])
            plan.append(dict(box=box, a=a, U=[e[1] for e in eig], lam3=lam3, s=s))
        return plan

    def fd_apply(self, r, plan):
        """z = P^{-1} r (fast_diagonalization_3d, tensor_algebra.f90:1107-1161,
        per component on its free box; zero on clamped dofs)."""
        r = np.asarray(r, dtype=np.float64).reshape(self.mask.shape)
        z = np.zeros_like(r)
        for c, pc in enumerate(plan):
            sl = tuple(slice(*pc["box"][d]) for d in (2, 1, 0))
            x = r[c][sl]
            if pc["s"] is not None:
                x = x * pc["s"]
            Uu, Uv, Uw = pc["U"]
            y = np.einsum("wvu,ua,vb,wc->cba", x, Uu, Uv, Uw, optimize=True)
            y = y / pc["lam3"]
            x = np.einsum("cba,ua,vb,wc->wvu", y, Uu, Uv, Uw, optimize=True)
            if pc["s"] is not None:
                x = x * pc["s"]
            z[c][sl] = x
        return z.ravel()

    def pcg(self, b, rtol=1e-8, maxit=10000, x0=None, precond=None):
        """Preconditioned CG (the loop of wq_mf_cg_3d, mf_wq_solver.f90:
        764-802 and 897-953), stopping on ||r||_2 <= rtol ||b||_2; Jacobi
        unless precond (a callable r -> z) is given.  Returns (x,
        iterations, rel. residual)."""
        m = self.mask.ravel()
        dinv = m / self.diag()
        if precond is None:
            precond = lambda v: dinv * v   # noqa: E731
        x = np.zeros_like(b) if x0 is None else x0.copy()
        r = (b - self.apply(x)) * m
        z = precond(r)
        p = z.copy()
        rz = r @ z
        bn = np.linalg.norm(b * m)
        it = 0
        for it in range(1, maxit + 1):
            Ap = self.apply(p)
            alpha = rz / (p @ Ap)
            x += alpha * p
            r -= alpha * Ap
            if np.linalg.norm(r) <= rtol * bn:
                break
            z = precond(r)
            rz_new = r @ z
            p = z + (rz_new / rz) * p
            rz = rz_new
        res = np.linalg.norm((b - self.apply(x)) * m) / bn
        return x, it, res
