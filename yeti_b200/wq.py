"""Weighted-quadrature matrix-free elasticity on the GPU.

``WQElasticity`` mirrors the reference's WQ driver
``iga_wq_mf/ThermoMechaIGA/pysrc/lib/fortran_mf_wq.py`` for the mechanical
problem: ``eval_Ku`` (``:404-419``), ``eval_bodyforce_vector`` (``:493-513``)
and ``mf_conj_grad`` (``:545-560``), on one NURBS patch with uniform open knot
vectors.  Everything runs in libyeti_b200.so (``yeti_wq_*``).

Vectors are component-major ``[c][iw][iv][iu]`` of length 3*ncp, clamped
dofs included and held at zero.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import CGStats, MEM_DEVICE, MEM_HOST, PREC_F32, PREC_F64, check, lib, ptr
from .patches import face_mask, free_mask

WQ_F64, WQ_F32 = 1, 2

# Preconditioners of yeti_wq_pcg (mode bits of include/yeti_b200.h).
PCG_FD, PCG_FD_SCALED, PCG_FD_UNIT, PCG_FD_TD = 4, 8, 16, 32
FD_VARIANTS = {
    "fd": PCG_FD,                        # a[c][d] = mean S[(c,d),(c,d)]
    "fd_scaled": PCG_FD | PCG_FD_SCALED,  # ... and sqrt(diag P / diag K)
    "fd_unit": PCG_FD | PCG_FD_UNIT,      # a[c][d] = 1
    "fd_td": PCG_FD | PCG_FD_TD,          # 1-D matrices weighted by the tensor
                                          # decomposition of the coefficients
    "fd_td_scaled": PCG_FD | PCG_FD_TD | PCG_FD_SCALED,
}
# The reference's Method strings of wq_mf_cg_3d (mf_wq_solver.f90:803-953).
REFERENCE_METHODS = {"WP": "jacobi", "C": "fd_unit", "JM": "fd", "JMS": "fd_scaled",
                     "TD": "fd_td", "TDS": "fd_td_scaled"}


def _precond_bits(precond):
    if precond == "jacobi":
        return 0
    if precond not in FD_VARIANTS:
        raise ValueError(f"precond {precond!r}: 'jacobi' or one of {sorted(FD_VARIANTS)}")
    return FD_VARIANTS[precond]


class WQElasticity:
    """WQ operator of a patch (see ``yeti_b200.patches.cube_patch``).

    clamp_faces: {'u0'|'u1'|'v0'|'v1'|'w0'|'w1': components} clamps those
    displacement components on the face (the reference erases the matching
    rows of its 1-D matrices, fortran_mf_wq.py:240-267).
    precisions: 'f64', 'f32' or 'both' operator data to keep on the device.
    """

    def __init__(self, patch, E, nu, clamp_faces=None, precisions="both",
                 ctx=None):
        self.ctx = ctx or _lib.default_context()
        self.patch = patch
        self.clamp_faces = clamp_faces or {}
        mask = {"f64": WQ_F64, "f32": WQ_F32, "both": WQ_F64 | WQ_F32}[precisions]
        p = np.ascontiguousarray(patch["p"], dtype=np.int32)
        nel = np.ascontiguousarray(patch["nel"], dtype=np.int32)
        # (3, ncp) in Fortran order: x, y, z of each control point together
        cps = np.ascontiguousarray(np.asarray(patch["cps"], dtype=np.float64).T)
        w = np.ascontiguousarray(patch["weights"], dtype=np.float64)
        dm = face_mask(self.clamp_faces)
        h = ctypes.c_void_p()
        check(lib().yeti_wq_setup(self.ctx.handle, ptr(p), ptr(nel), ptr(cps),
                                  ptr(w), float(E), float(nu), ptr(dm), mask,
                                  ctypes.byref(h)), "yeti_wq_setup")
        self.handle = h
        vals = [ctypes.c_int64() for _ in range(5)]
        check(lib().yeti_wq_info(h, *[ctypes.byref(v) for v in vals]),
              "yeti_wq_info")
        self.ncp, self.ndof, self.nfree, self.nqp, self.bytes = (v.value for v in vals)
        self.free_mask = free_mask(patch, self.clamp_faces)

    @classmethod
    def from_iga_model(cls, modelIGA, mechablockedboundaries=None, E=None, nu=None,
                       ipatch=0, precisions="both", ctx=None):
        """The operator of patch ipatch (0-based) of a YETI IGAparametrization,
        as ``fortran_mf_wq(modelIGA, isThermal=False, isMechanical=True,
        mechablockedboundaries=...)`` builds it (fortran_mf_wq.py:31-71):
        mechablockedboundaries = [[u0, u1], [v0, v1], [w0, w1]] face flags
        (default all blocked, as the reference), E and nu from the patch's
        ``_MATERIAL_PROPERTIES`` unless given.  ``cp_index`` keeps the model
        control point of every tensor position (``to_model_layout``)."""
        from .patches import clamp_faces_from_blocked, patch_from_iga_model
        patch, cp_index = patch_from_iga_model(modelIGA, ipatch)
        mat = np.asarray(modelIGA._MATERIAL_PROPERTIES, dtype=np.float64).reshape(2, -1)
        E = float(mat[0, ipatch]) if E is None else float(E)
        nu = float(mat[1, ipatch]) if nu is None else float(nu)
        if mechablockedboundaries is None:
            mechablockedboundaries = [[1, 1], [1, 1], [1, 1]]
        op = cls(patch, E, nu, clamp_faces_from_blocked(mechablockedboundaries),
                 precisions=precisions, ctx=ctx)
        op.cp_index = cp_index
        op.nb_cp_model = int(modelIGA._nb_cp)
        return op

    def to_model_layout(self, x):
        """A component-major WQ vector as the model's (3, nb_cp) array (the
        layout of YETI's solution writers); model control points outside
        the patch are 0."""
        out = np.zeros((3, self.nb_cp_model))
        out[:, self.cp_index] = np.asarray(x, dtype=np.float64).reshape(3, -1)
        return out

    def from_model_layout(self, U):
        """The model's (3, nb_cp) (or interleaved nb_dof) array as a
        component-major WQ vector of this patch."""
        U = np.asarray(U, dtype=np.float64)
        if U.ndim == 1:
            U = U.reshape(-1, 3).T
        return np.ascontiguousarray(U[:, self.cp_index]).ravel()

    # ------------------------------------------------------------- operator
    def eval_Ku(self, u, precision="f64"):
        """K u.  u: numpy array (host) or torch CUDA tensor (device, result
        returned as a tensor of the same dtype)."""
        prec = PREC_F64 if precision == "f64" else PREC_F32
        if isinstance(u, np.ndarray):
            dt = np.float64 if prec == PREC_F64 else np.float32
            uu = np.ascontiguousarray(u, dtype=dt)
            out = np.empty_like(uu)
            check(lib().yeti_wq_apply(self.handle, ptr(uu), ptr(out), prec,
                                      MEM_HOST), "yeti_wq_apply")
            return out
        import torch
        uu = u.contiguous()
        out = torch.empty_like(uu)
        check(lib().yeti_wq_apply(self.handle, ptr(uu), ptr(out), prec,
                                  MEM_DEVICE), "yeti_wq_apply")
        return out

    def apply_device(self, u, out, precision="f64"):
        """out = K u for device tensors (no allocation, no host sync)."""
        prec = PREC_F64 if precision == "f64" else PREC_F32
        check(lib().yeti_wq_apply(self.handle, ptr(u), ptr(out), prec,
                                  MEM_DEVICE), "yeti_wq_apply")

    def diag(self):
        d = np.empty(self.ndof)
        check(lib().yeti_wq_diag(self.handle, ptr(d), MEM_HOST), "yeti_wq_diag")
        return d

    def eval_bodyforce_vector(self, f):
        """Load vector of a constant body-force density f = (fx, fy, fz)."""
        ff = np.ascontiguousarray(f, dtype=np.float64)
        out = np.empty(self.ndof)
        check(lib().yeti_wq_body_force(self.handle, ptr(ff), ptr(out),
                                       MEM_HOST), "yeti_wq_body_force")
        return out

    # --------------------------------------------------------------- solver
    def pcg(self, b, rtol=1e-8, maxit=20000, mixed=False, x0=None,
            method="cg", precond="jacobi"):
        """Preconditioned Krylov solve of K x = b.

        method 'cg' (mf_wq_solver.f90:764-802) or 'bicgstab'
        (mf_wq_solver.f90:958-1308).  mixed=True: FP32 operator and Krylov
        vectors with the FP64 true residual (CG: reliable updates; BiCGSTAB:
        iterative refinement).  precond: 'jacobi' or a fast-diagonalisation
        variant of FD_VARIANTS (mf_wq_solver.f90:803-953).  b, x0: numpy
        (host) or torch CUDA float64 tensors.  Returns (x, stats dict)."""
        st = CGStats()
        mode = (1 if mixed else 0) | (2 if method == "bicgstab" else 0)
        mode |= _precond_bits(precond)
        if isinstance(b, np.ndarray):
            bb = np.ascontiguousarray(b, dtype=np.float64)
            x = np.zeros_like(bb) if x0 is None else np.array(x0, dtype=np.float64)
            mem = MEM_HOST
        else:
            import torch
            bb = b.contiguous()
            x = torch.zeros_like(bb) if x0 is None else x0.clone()
            mem = MEM_DEVICE
        rc = lib().yeti_wq_pcg(self.handle, ptr(bb), ptr(x), float(rtol),
                               int(maxit), mode, ctypes.byref(st), mem)
        check(rc, "yeti_wq_pcg")
        return x, st.as_dict()

    def fd_apply(self, r, precond="fd_scaled", prec=PREC_F64):
        """z = P^{-1} r for a fast-diagonalisation variant of FD_VARIANTS
        (numpy host arrays: float64 for PREC_F64, float32 for PREC_F32)."""
        if precond not in FD_VARIANTS:
            raise ValueError(f"precond {precond!r}: one of {sorted(FD_VARIANTS)}")
        dt = np.float64 if prec == PREC_F64 else np.float32
        rr = np.ascontiguousarray(r, dtype=dt)
        z = np.empty_like(rr)
        check(lib().yeti_wq_fd_apply(self.handle, ptr(rr), ptr(z), prec,
                                     FD_VARIANTS[precond], MEM_HOST),
              "yeti_wq_fd_apply")
        return z

    def mf_conj_grad(self, bi, nbIterations, epsilon, method="WP",
                     directsol=None, isCG=True):
        """Twin of fortran_mf_wq.mf_conj_grad (fortran_mf_wq.py:545-560):
        returns (sol, residue, error) with the reference's per-iteration
        histories RelRes(k) = max|r_k| / max|b| and RelError(k) =
        max|directsol - x_k| / max|directsol| (zeros without directsol),
        k = 0..iterations, stopping when RelRes <= epsilon
        (wq_mf_cg_3d / wq_mf_bicgstab_3d, mf_wq_solver.f90:642-1308).
        method: 'WP' (Jacobi) or the fast-diagonalisation forms 'C', 'JM',
        'JMS', 'TD', 'TDS' (mf_wq_solver.f90:803-953, per displacement
        component).  FP64 throughout, as the reference."""
        if method not in REFERENCE_METHODS:
            raise NotImplementedError(
                f"method {method!r}: supported {sorted(REFERENCE_METHODS)}")
        mode = (0 if isCG else 2) | _precond_bits(REFERENCE_METHODS[method])
        bb = np.ascontiguousarray(bi, dtype=np.float64)
        x = np.zeros_like(bb)
        maxit = int(nbIterations)
        relres = np.zeros(maxit + 1)
        relerr = np.zeros(maxit + 1)
        ds = None if directsol is None else np.ascontiguousarray(directsol, dtype=np.float64)
        st = CGStats()
        rc = lib().yeti_wq_pcg_history(self.handle, ptr(bb), ptr(x), float(epsilon), maxit,
                                       mode, ptr(ds) if ds is not None else None,
                                       ptr(relres), ptr(relerr), ctypes.byref(st), MEM_HOST)
        check(rc, "yeti_wq_pcg_history")
        k = int(st.iterations)
        self.last_stats = st.as_dict()
        return x, relres[:k + 1], relerr[:k + 1]

    def close(self):
        if getattr(self, "handle", None):
            lib().yeti_wq_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
