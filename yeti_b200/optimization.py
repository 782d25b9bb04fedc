"""Shape-optimisation responses of a U1 solid model, evaluated on the GPU.

``ShapeOptimization`` mirrors the response API of the reference's
``IgaOptimization`` (``src/yeti_iga/overlay/iga_optimization.py:18-221``) and
the ``OPTmodelling`` functions behind it
(``preprocessing/igaparametrization/OPT_modelling.py:164-235, 411-445,
508-565``):

* ``volume`` / ``grad_volume_analytic`` / ``grad_volume_finite_differences``
  (``iga_optimization.py:69-159``, ``OPT_modelling.py:508-531``);
* ``compliance`` / ``grad_compliance_analytic`` /
  ``grad_compliance_finite_differences`` (``iga_optimization.py:162-221``,
  ``OPT_modelling.py:534-565``): C = 1/2 U.F, adjoint U_A = U/2,
  dC/dP = dW_int + 2 dW_ext;
* ``displacement`` / ``grad_displacement_analytic`` /
  ``grad_displacement_finite_differences`` (``iga_optimization.py:223-298``,
  ``OPT_modelling.py:568-608``): u(xi) = sum_a R_a(xi) U_a, one adjoint per
  component with the right-hand side R_a(xi) on that component's dofs
  (``adjointRHSdisp``, ``optim/adjointRHS_disp.f:19-100``),
  du_c/dP = dW_int + dW_ext of adjoint c.

The design variables x move the design model's control points through
``update_function(coords_0, x) -> coords`` (3, nb_cp_design); the analysis
model's control points are ``coarse_to_fine @ coords.T`` (the reference's
``_mapCoarse2Fine``, a fixed linear map: knot insertion and degree elevation
in homogeneous coordinates divided by the fine weights), or the design
points themselves when no map is given.  Gradients are propagated back as in
``_propagateSensitivityAnalysis`` (``OPT_modelling.py:439-445``): the fine
gradient through the transposed map, then contracted with
d coords / d x_i from ``d_update_function(coords_0, x, i)`` or, when none is
given, central differences of ``update_function``.

Every response runs the GPU kernels of libyeti_b200.so: the COO assembly
(``yeti_assemble_u1_coo``), the adjoint shape gradient
(``yeti_grad_lin_elast_work``) and the volume kernels (``yeti_volume_u1``);
the free-dof system is solved directly on the host, as the reference does.
The reference's ``update_function`` edits an ``IgaModel`` in place; here it
returns the new coordinates, and the refinement is given as the matrix the
reference builds from its ``Refinement``.  The rational basis at the point
of a displacement response is evaluated on the host (one element's
(p+1)^3 values, as the reference does); VTU output stays with YETI's
writers.
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .gradient import _solve, grad_from_system_args
from .stiffmtrx_elemstorage import SYSTEM_ARG_NAMES, sys_linmat_lindef_static
from .volume import volume_and_gradient

__all__ = ["ShapeOptimization"]


class ShapeOptimization:
    """Volume and compliance of a U1 model as functions of design variables.

    Parameters
    ----------
    system_args : list
        The analysis model's 38 arguments of ``sys_linmat_lindef_static``
        (``IGAparametrization.get_inputs4system_elemStorage``).
    nb_var : int
        Number of design variables.
    update_function : callable
        ``update_function(coords_0, x)`` returns the design control points
        (3, nb_cp_design) for the design variables x.
    coords_0 : array (3, nb_cp_design), optional
        Initial design control points; default: the analysis model's.
    coarse_to_fine : array or sparse matrix (nb_cp, nb_cp_design), optional
        Linear map from design to analysis control points; default identity.
    d_update_function : callable, optional
        ``d_update_function(coords_0, x, ivar)`` returns d coords / d x_ivar
        (3, nb_cp_design).
    include_surface_loads : bool
        Add the sensitivity of surface loads on moving faces to the analytic
        compliance gradient (the reference leaves it out; default False keeps
        its values).
    """

    def __init__(self, system_args, nb_var, update_function, coords_0=None,
                 coarse_to_fine=None, d_update_function=None,
                 include_surface_loads=False, ctx=None):
        if len(system_args) != len(SYSTEM_ARG_NAMES):
            raise ValueError(f"system_args has {len(system_args)} entries, "
                             f"expected {len(SYSTEM_ARG_NAMES)}")
        self.args = list(system_args)
        self._d = dict(zip(SYSTEM_ARG_NAMES, self.args))
        self.nb_var = int(nb_var)
        self.update_function = update_function
        self.d_update_function = d_update_function
        self.include_surface_loads = bool(include_surface_loads)
        self.ctx = ctx
        fine0 = np.asarray(self._d["COORDS3D"], dtype=np.float64)
        self.nb_cp = fine0.shape[1]
        self.coords_0 = (fine0.copy() if coords_0 is None
                         else np.array(coords_0, dtype=np.float64))
        if self.coords_0.ndim != 2 or self.coords_0.shape[0] != 3:
            raise ValueError("coords_0 must have shape (3, nb_cp_design)")
        if coarse_to_fine is None:
            if self.coords_0.shape[1] != self.nb_cp:
                raise ValueError("without coarse_to_fine the design model must have "
                                 "the analysis model's control points")
            self.map = None
        else:
            self.map = sp.csr_matrix(coarse_to_fine, dtype=np.float64)
            if self.map.shape != (self.nb_cp, self.coords_0.shape[1]):
                raise ValueError(f"coarse_to_fine has shape {self.map.shape}, expected "
                                 f"({self.nb_cp}, {self.coords_0.shape[1]})")
        self.nb_patch = int(np.atleast_1d(self._d["nb_elem_patch"]).size)
        self._cache_x = None
        self._cache_sol = None
        self._tables = None

    # ------------------------------------------------------------ geometry
    def _check_x(self, x):
        x = np.asarray(x, dtype=np.float64).ravel()
        if x.size != self.nb_var:
            raise ValueError(f"x has {x.size} entries, expected {self.nb_var}")
        return x

    def design_coords(self, x):
        """Design control points (3, nb_cp_design) for x."""
        c = np.asarray(self.update_function(self.coords_0.copy(), self._check_x(x)),
                       dtype=np.float64)
        if c.shape != self.coords_0.shape:
            raise ValueError(f"update_function returned shape {c.shape}, "
                             f"expected {self.coords_0.shape}")
        return c

    def analysis_coords(self, x):
        """Analysis control points (3, nb_cp) for x (_mapCoarse2Fine,
        OPT_modelling.py:187-225)."""
        c = self.design_coords(x)
        if self.map is None:
            return c
        return np.ascontiguousarray((self.map @ c.T).T)

    def _d_design(self, x, ivar):
        if self.d_update_function is not None:
            d = np.asarray(self.d_update_function(self.coords_0.copy(), x, ivar),
                           dtype=np.float64)
            if d.shape != self.coords_0.shape:
                raise ValueError(f"d_update_function returned shape {d.shape}, "
                                 f"expected {self.coords_0.shape}")
            return d
        h = 1e-6 * max(1.0, abs(x[ivar]))
        xp, xm = x.copy(), x.copy()
        xp[ivar] += h
        xm[ivar] -= h
        return (self.design_coords(xp) - self.design_coords(xm)) / (2.0 * h)

    def propagate(self, x, grad_fine):
        """d response / d x from d response / d P_fine (3, nb_cp)
        (_propagateSensitivityAnalysis, OPT_modelling.py:439-445)."""
        x = self._check_x(x)
        g = np.asarray(grad_fine, dtype=np.float64)
        g_design = g if self.map is None else np.asarray((self.map.T @ g.T).T)
        return np.array([np.tensordot(self._d_design(x, i), g_design, axes=2)
                         for i in range(self.nb_var)])

    def _listpatch(self, listpatch):
        if listpatch is None:
            return np.ones(self.nb_patch, dtype=np.int64)
        lp = np.atleast_1d(np.asarray(listpatch))
        if lp.size != self.nb_patch:
            raise ValueError(f"Length of listpatch parameter must be equal to {self.nb_patch}")
        if not np.all(np.isin(lp, [0, 1])):
            raise ValueError("listpatch parameters must exclusively contain 0 or 1 values.")
        return lp.astype(np.int64)

    def _area_inputs(self, coords, listpatch):
        d = self._d
        return [self._listpatch(listpatch), coords, d["IEN"], d["nb_elem_patch"], d["Nkv"],
                d["Ukv"], d["Nijk"], d["weight"], d["Jpqr"], d["ELT_TYPE"], d["PROPS"],
                d["JPROPS"], d["TENSOR"], d["MCRD"], d["NBINT"], d["NNODE"]]

    # ------------------------------------------------------------ responses
    def volume(self, x, listpatch=None):
        """Volume of the listed patches (all by default) at x."""
        v, _ = volume_and_gradient(self._area_inputs(self.analysis_coords(x), listpatch),
                                   gradient=False, ctx=self.ctx)
        return v

    def grad_volume_analytic(self, x, listpatch=None):
        """dV/dx from the GPU volume gradient."""
        _, g = volume_and_gradient(self._area_inputs(self.analysis_coords(x), listpatch),
                                   gradient=True, ctx=self.ctx)
        return self.propagate(x, g)

    def grad_volume_finite_differences(self, x, eps=1.e-6, centered=False, listpatch=None):
        return self._sensitivity_fd(lambda y: self.volume(y, listpatch), x, eps, centered)

    def _state(self, x):
        x = self._check_x(x)
        if self._cache_x is None or not np.array_equal(self._cache_x, x):
            X = self.analysis_coords(x)
            U, F = _solve(self.args, X)
            self._cache_x, self._cache_sol = x.copy(), (X, U, F)
        return self._cache_sol

    def compliance(self, x):
        """Discrete compliance 1/2 U.F at x (compute_compliance_discrete)."""
        _, U, F = self._state(x)
        return 0.5 * float(U @ F)

    def grad_compliance_analytic(self, x):
        """dC/dx: adjoint U/2 on the GPU, dW_int + 2 dW_ext, propagated."""
        X, U, _ = self._state(x)
        a = list(self.args)
        a[2] = X
        sol = U.reshape(-1, 3).T
        gi, ge = grad_from_system_args(a, sol, 0.5 * sol[None], True, True,
                                       self.include_surface_loads)
        return self.propagate(x, gi[0] + 2.0 * ge[0])

    def grad_compliance_finite_differences(self, x, eps=1.e-6, centered=False):
        return self._sensitivity_fd(self.compliance, x, eps, centered)

    def _sensitivity_fd(self, fun, x, eps, centered):
        """Forward or central differences per design variable
        (_sensitivityFD, OPT_modelling.py:411-437): shape (nb_var,) for a
        scalar response, (nb_var, m) for a response of m values."""
        x = self._check_x(x)
        f = lambda y: np.asarray(fun(y), dtype=np.float64)
        f0 = None if centered else f(x)
        rows = []
        for i in range(self.nb_var):
            xp = x.copy()
            xp[i] += eps
            if centered:
                xm = x.copy()
                xm[i] -= eps
                rows.append((f(xp) - f(xm)) / (2.0 * eps))
            else:
                rows.append((f(xp) - f0) / eps)
        return np.array(rows)

    # ------------------------------------------------------------ displacement
    def _patch_tables(self):
        """Per patch: element count, knot counts, degrees, nodes per
        element, and the offsets of its first element, of its nodes in the
        flat IEN / weight arrays and of its knots in Ukv."""
        if self._tables is None:
            d = self._d
            nep = np.atleast_1d(np.asarray(d["nb_elem_patch"], dtype=np.int64))
            nkv = np.asarray(d["Nkv"], dtype=np.int64).reshape(3, -1, order="F")
            jpqr = np.asarray(d["Jpqr"], dtype=np.int64).reshape(3, -1, order="F")
            nnode = np.atleast_1d(np.asarray(d["NNODE"], dtype=np.int64))
            e0 = np.concatenate([[0], np.cumsum(nep)[:-1]])
            n0 = np.concatenate([[0], np.cumsum(nep * nnode)[:-1]])
            k0 = np.concatenate([[0], np.cumsum(nkv.sum(axis=0))[:-1]])
            nijk = np.asarray(d["Nijk"], dtype=np.int64).reshape(3, -1, order="F")
            self._tables = (nep, nkv, jpqr, nnode, e0, n0, k0, nijk)
        return self._tables

    def point_basis(self, xi, ipatch=0):
        """Control points (0-based) and rational basis values R of the
        element of patch ipatch holding the parametric point xi
        (updateElementNumber + evalnurbs, evaluatenurbsfcts.f:94-209): the
        knot span of each coordinate (the last non-empty one at the end of
        the knot vector), the element with those spans (Nijk), the reversed
        tensor product of the B-spline values times the element's weights,
        divided by their sum.  ipatch is 0-based: the reference's 1-based
        numpatch minus one."""
        nep, nkv, jpqr, nnode, e0, n0, k0, nijk = self._patch_tables()
        if not 0 <= ipatch < nep.size:
            raise ValueError(f"ipatch {ipatch} outside 0..{nep.size - 1}")
        xi = np.asarray(xi, dtype=np.float64).ravel()
        if xi.size != 3:
            raise ValueError("xi must hold 3 parametric coordinates")
        U = np.asarray(self._d["Ukv"], dtype=np.float64).ravel()
        off = int(k0[ipatch])
        spans, vals = [], []
        for dd in range(3):
            kv = U[off:off + nkv[dd, ipatch]]
            off += int(nkv[dd, ipatch])
            p = int(jpqr[dd, ipatch])
            u = float(xi[dd])
            if not kv[0] <= u <= kv[-1]:
                raise ValueError(f"xi[{dd}] = {u} outside [{kv[0]}, {kv[-1]}]")
            ni = min(int(np.searchsorted(kv, u, side="right")), kv.size - p - 1)
            # Cox-de Boor on span [kv[ni-1], kv[ni]] (The NURBS Book A2.2)
            N = np.zeros(p + 1)
            N[0] = 1.0
            left, right = np.zeros(p + 1), np.zeros(p + 1)
            for j in range(1, p + 1):
                left[j] = u - kv[ni - j]
                right[j] = kv[ni + j - 1] - u
                saved = 0.0
                for r in range(j):
                    temp = N[r] / (right[r + 1] + left[j - r])
                    N[r] = saved + right[r + 1] * temp
                    saved = left[j - r] * temp
                N[j] = saved
            spans.append(ni)
            vals.append(N[::-1])   # local node i <-> function p - i
        first, count = int(e0[ipatch]), int(nep[ipatch])
        hit = np.nonzero(np.all(nijk[:, first:first + count] == np.array(spans)[:, None],
                                axis=0))[0]
        if hit.size == 0:
            raise ValueError(f"no element of patch {ipatch} holds xi = {xi}")
        le = int(hit[0])
        nn = int(nnode[ipatch])
        base = int(n0[ipatch]) + le * nn
        w = np.asarray(self._d["weight"], dtype=np.float64).ravel()[base:base + nn]
        cps = np.asarray(self._d["IEN"], dtype=np.int64).ravel()[base:base + nn] - 1
        R = (vals[2][:, None, None] * vals[1][None, :, None] * vals[0][None, None, :]).ravel() * w
        return cps, R / R.sum()

    def displacement(self, x, xi, ipatch=0):
        """Displacement (3,) at the parametric point xi of patch ipatch
        (compute_displacement, OPT_modelling.py:568-576).  ipatch is 0-based:
        the reference's numpatch (1-based, default 1) minus one."""
        _, U, _ = self._state(x)
        cps, R = self.point_basis(xi, ipatch)
        return R @ U.reshape(-1, 3)[cps]

    def grad_displacement_analytic(self, x, xi, ipatch=0):
        """du/dx, shape (nb_var, 3): three adjoint solves with the point's
        basis on each component, the GPU adjoint kernel with three adjoints,
        dW_int + dW_ext per component, propagated
        (compute_gradDisplacement_AN, OPT_modelling.py:595-608).  ipatch is
        0-based (the reference's numpatch - 1)."""
        X, U, _ = self._state(x)
        cps, R = self.point_basis(xi, ipatch)
        n = U.size
        FA = np.zeros((n, 3))
        for c in range(3):
            FA[3 * cps + c, c] = R
        a = list(self.args)
        a[2] = X
        kdata, krow, kcol, _ = sys_linmat_lindef_static(*a)
        K = sp.coo_matrix((kdata, (krow, kcol)), shape=(n, n)).tocsc()
        K = K + K.T
        idof = np.asarray(self.args[26])[:int(self.args[27])] - 1
        UA = np.zeros((n, 3))
        UA[idof] = np.asarray(spla.spsolve(K[idof, :][:, idof], FA[idof])).reshape(-1, 3)
        sol = U.reshape(-1, 3).T
        adj = np.stack([UA[:, c].reshape(-1, 3).T for c in range(3)])
        gi, ge = grad_from_system_args(a, sol, adj, True, True, self.include_surface_loads)
        return np.stack([self.propagate(x, gi[c] + ge[c]) for c in range(3)], axis=1)

    def grad_displacement_finite_differences(self, x, xi, ipatch=0, eps=1.e-6,
                                             centered=False):
        """du/dx by differences, shape (nb_var, 3); ipatch 0-based."""
        return self._sensitivity_fd(lambda y: self.displacement(y, xi, ipatch), x, eps,
                                    centered)
