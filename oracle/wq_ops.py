"""FP64 numpy oracle of the weighted-quadrature (WQ) elastic operator on a
single NURBS patch.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

The reference ships the WQ matrix-free operator for the scalar (thermal)
problem only, with B-spline geometry:
  * K u = sum_{k,l} W^{(k,l)} (coef_kl * (B^{(l)})^T u)
    (mf_wq_get_ku_3d, src/yeti_iga/iga_wq_mf/fsrc/mf_wq_solver.f90:284-544),
    W^{(k,l)} the Kronecker product of the 1-D weights W^{[d==k][d==l]};
  * the elastic coefficient S = ext(invJ)^T (MM^T DD MM) ext(invJ) detJ
    (eval_mech_coefficient, wq_assembly.f90:52-138) used per 3x3 component
    block (wq_get_stiffness_3d, wq_assembly.f90:1020-1054);
  * the Jacobian from B-spline sums (jacobien_physicalposition_3d,
    wq_assembly.f90:233-473).
This oracle composes them into the elastic operator and extends it to NURBS:

  u_j = v_j / W with v_j = sum_a N_a (w_a U_aj), W = sum_a N_a w_a, and the
  test function R_a = w_a N_a / W, so that with S^ = S / W^2, g = grad W / W

      (K U)_ai = w_a sum_{kappa,lambda} sum_q W^{kappa,lambda}_a(q) H^{kappa,lambda}_i(q)

  over test kinds kappa (0: value, 1..3: derivative direction) and trial
  kinds lambda (same), with, at each point,
      H^{k,l}_i = sum_j S^[(i,k),(j,l)] dv_j/dxi_l
      H^{k,0}_i = -sum_j (sum_l S^[(i,k),(j,l)] g_l) v_j
      H^{0,lambda}_i = -sum_k g_k H^{k,lambda}_i .
  The 1-D weight of direction d is W^{[d==kappa][d==lambda]} (test order,
  trial order), as in the reference.  With all weights 1, g = 0 and this is
  exactly the reference's operator per component block.

Two deliberate differences from the reference's code, both documented in
DESIGN.md: the coefficient uses the geometric orientation
S = ext(invJ) MDM ext(invJ)^T |detJ| with invJ = (dx/dxi)^{-1} (the
reference's product is transposed, which only agrees for symmetric
Jacobians), and the Jacobian includes the NURBS weights.
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
    """(nw, nv, nu) field on functions -> (qw, qv, qu) values at points."""
    t = np.einsum("wvu,uq->wvq", f, Bu)
    t = np.einsum("wvq,vr->wrq", t, Bv)
    return np.einsum("wrq,ws->srq", t, Bw)


def _bwd(h, Wu, Wv, Ww):
    """(qw, qv, qu) point values -> (nw, nv, nu) with the 1-D weights."""
    t = np.einsum("srq,uq->sru", h, Wu)
    t = np.einsum("sru,vr->svu", t, Wv)
    return np.einsum("svu,ws->wvu", t, Ww)


class WQOracle:
    """FP64 WQ elasticity on one patch (see module docstring)."""

    def __init__(self, patch, E, nu, clamp_faces=None):
        from yeti_b200.patches import free_mask
        self.p = tuple(patch["p"])
        self.nel = tuple(patch["nel"])
        self.n = [self.p[d] + self.nel[d] for d in range(3)]
        self.rules = [wq_rules.wq_rule(self.p[d], self.nel[d]) for d in range(3)]
        nu_, nv_, nw_ = self.n
        self.w = patch["weights"].reshape(nw_, nv_, nu_)
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
        self.detJ = np.linalg.det(Jq)
        invJ = np.linalg.inv(Jq)                  # invJ[..., k, d] = dxi_k/dx_d
        MDM = mdm_matrix(E, nu)
        P = np.zeros(Jq.shape[:-2] + (9, 9))
        for c in range(3):
            P[..., 3 * c:3 * c + 3, 3 * c:3 * c + 3] = invJ
        S = P @ MDM @ np.swapaxes(P, -1, -2) * np.abs(self.detJ)[..., None, None]
        self.Shat = S / (W ** 2)[..., None, None]  # (..., 9, 9)
        self.g = np.moveaxis(gW / W, 0, -1)         # (..., 3)
        self.W = W
        self.x = x

    # ------------------------------------------------------------ operator
    def _H(self, F, i):
        """The 16 point fields H^{kappa,lambda}_i, keyed (kappa, lambda)."""
        Sh, g = self.Shat, self.g
        H = {}
        for k in (1, 2, 3):
            for l in (1, 2, 3):
                H[k, l] = sum(Sh[..., 3 * i + k - 1, 3 * j + l - 1] * F[l][j]
                              for j in range(3))
            A = [sum(Sh[..., 3 * i + k - 1, 3 * j + l - 1] * g[..., l - 1]
                     for l in (1, 2, 3)) for j in range(3)]
            H[k, 0] = -sum(A[j] * F[0][j] for j in range(3))
        for lam in range(4):
            H[0, lam] = -sum(g[..., k - 1] * H[k, lam] for k in (1, 2, 3))
        return H

    def apply(self, u):
        u = np.asarray(u, dtype=np.float64).reshape(self.mask.shape) * self.mask
        v = [self.w * u[j] for j in range(3)]
        F = [[self.fwd(v[j], lam) for j in range(3)] for lam in range(4)]
        out = np.zeros_like(u)
        for i in range(3):
            H = self._H(F, i)
            acc = 0.0
            for (kap, lam), h in H.items():
                acc = acc + self.bwd(h, kap, lam)
            out[i] = self.w * acc
        return (out * self.mask).ravel()

    def diag(self):
        Sh, g = self.Shat, self.g
        out = np.zeros(self.mask.shape)
        for i in range(3):
            acc = 0.0
            for kap in range(4):
                for lam in range(4):
                    if kap and lam:
                        C = Sh[..., 3 * i + kap - 1, 3 * i + lam - 1]
                    elif kap:
                        C = -sum(Sh[..., 3 * i + kap - 1, 3 * i + l - 1] * g[..., l - 1]
                                 for l in (1, 2, 3))
                    elif lam:
                        C = -sum(g[..., k - 1] * Sh[..., 3 * i + k - 1, 3 * i + lam - 1]
                                 for k in (1, 2, 3))
                    else:
                        C = sum(g[..., k - 1] * Sh[..., 3 * i + k - 1, 3 * i + l - 1] * g[..., l - 1]
                                for k in (1, 2, 3) for l in (1, 2, 3))
                    mats = [self._W(d, kap == d + 1, lam == d + 1) *
                            self._B(d, lam == d + 1) for d in range(3)]
                    acc = acc + _bwd(C, *mats)
            out[i] = self.w ** 2 * acc
        out = np.where(self.mask > 0, out, 1.0)
        return out.ravel()

    def body_force(self, f):
        """Load vector of a constant force density f (wq_get_force_3d,
        wq_assembly.f90:1193-1251, with the rational test functions)."""
        out = np.zeros(self.mask.shape)
        for i in range(3):
            h = f[i] * np.abs(self.detJ) / self.W
            out[i] = self.w * self.bwd(h, 0, 0)
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

    def pcg(self, b, rtol=1e-8, maxit=10000, x0=None):
        """Jacobi-preconditioned CG (the 'WP' loop of wq_mf_cg_3d,
        mf_wq_solver.f90:764-802, with a Jacobi preconditioner), stopping on
        ||r||_2 <= rtol ||b||_2.  Returns (x, iterations, rel. residual)."""
        m = self.mask.ravel()
        dinv = m / self.diag()
        x = np.zeros_like(b) if x0 is None else x0.copy()
        r = (b - self.apply(x)) * m
        z = dinv * r
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
            z = dinv * r
            rz_new = r @ z
            p = z + (rz_new / rz) * p
            rz = rz_new
        res = np.linalg.norm((b - self.apply(x)) * m) / bn
        return x, it, res
