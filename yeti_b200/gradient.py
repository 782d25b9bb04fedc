"""Adjoint shape gradient of the linear-elastic work (U1 solids) on the GPU.

``gradlinelastwork_an`` is the drop-in for the reference's
``optim.gradadjointwork.gradlinelastwork_an`` (called at
``preprocessing/igaparametrization/OPT_modelling.py:474-477`` with the list of
``IGAparametrization._get_inputs4gradTotalwork``, ``IGA_parametrization.py:
1507-1527``); it runs ``yeti_grad_lin_elast_work`` in libyeti_b200.so.

``Compliance`` is a ``torch.autograd.Function`` for the discrete compliance
C(P) = 1/2 U.F with K(P) U = F(P): the forward pass assembles on the GPU and
solves the free dofs directly; the backward pass runs the adjoint kernel
(U_A = U/2, dC/dP = dW_int + 2 dW_ext, as in
``OPTmodelling.compute_gradCompliance_AN``, ``OPT_modelling.py:558-565``),
which recomputes the quadrature-point geometry from the control points.
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import _lib
from ._lib import MEM_HOST, check, lib, ptr
from .stiffmtrx_elemstorage import pack_u1_model, sys_linmat_lindef_static

__all__ = ["gradlinelastwork_an", "grad_from_system_args", "Compliance",
           "compliance_and_gradient"]


def gradlinelastwork_an(computeWint, computeWext, sol, ADJ, activeElem,
                        activeDir, COORDS, IEN, nb_elem_patch, Nkv, Ukv, Nijk,
                        weight, Jpqr, ELT_TYPE, PROPS, JPROPS,
                        MATERIAL_PROPERTIES, RHO, TENSOR, indDLoad, JDLType,
                        ADLMAG, load_target_nbelem, load_additionalInfos,
                        NBPINT, nnode, nadj=None, mcrd=3, nb_load=None,
                        nb_patch=None, nb_elem=None, nb_cp=None,
                        include_surface_loads=False, ctx=None):
    """GPU twin of gradadjointwork.gradlinelastwork_an
    (gradtotalwork_fullAN.f90:17-300).  Returns (gradWint, gradWext), each of
    shape (nadj, 3, nb_cp).  include_surface_loads=False reproduces the
    reference (which leaves the surface-load term out,
    gradUELMAT_solid.f90:463-477); True adds it."""
    coords = np.asarray(COORDS, dtype=np.float64)
    nbl = len(np.atleast_1d(JDLType))
    args = [activeElem, 0, coords, IEN, nb_elem_patch, Nkv, Ukv, Nijk, weight,
            Jpqr, ELT_TYPE, PROPS, JPROPS, MATERIAL_PROPERTIES, None, RHO,
            TENSOR, indDLoad, JDLType, ADLMAG, load_target_nbelem,
            load_additionalInfos, np.zeros(nbl, dtype=np.int64), None, None,
            None, None, None, mcrd, NBPINT, nnode, np.zeros((1, coords.shape[1]))]
    return grad_from_system_args(args, np.asarray(sol), np.asarray(ADJ),
                                 bool(computeWint), bool(computeWext),
                                 include_surface_loads, ctx)


def grad_from_system_args(args, sol, adj, compute_int=True, compute_ext=True,
                          include_surface=False, ctx=None):
    """Gradient for a model given as the argument list of
    sys_linmat_lindef_static.  sol: (3, nb_cp); adj: (nadj, 3, nb_cp)."""
    pm = pack_u1_model(*args[:32])
    ctx = ctx or _lib.default_context()
    nb_cp = pm.struct.nb_cp
    sol = np.ascontiguousarray(np.asarray(sol, dtype=np.float64).T)       # (nb_cp, 3)
    adj = np.asarray(adj, dtype=np.float64)
    nadj = adj.shape[0]
    adjf = np.ascontiguousarray(np.transpose(adj, (2, 1, 0)))            # Fortran (nadj,3,ncp)
    gi = np.zeros((nb_cp, 3, nadj))
    ge = np.zeros((nb_cp, 3, nadj))
    check(lib().yeti_grad_lin_elast_work(
        ctx.handle, pm.struct, ptr(sol), ptr(adjf), nadj, int(compute_int),
        int(compute_ext), int(include_surface), ptr(gi), ptr(ge), MEM_HOST),
        "yeti_grad_lin_elast_work")
    return np.transpose(gi, (2, 1, 0)).copy(), np.transpose(ge, (2, 1, 0)).copy()


def _solve(args, coords):
    a = list(args)
    a[2] = coords
    kdata, krow, kcol, F = sys_linmat_lindef_static(*a)
    n = F.size
    K = sp.coo_matrix((kdata, (krow, kcol)), shape=(n, n)).tocsc()
    K = K + K.T
    nfree = int(args[27])
    idof = np.asarray(args[26])[:nfree] - 1
    U = np.zeros(n)
    U[idof] = spla.spsolve(K[idof, :][:, idof], F[idof])
    return U, F


def compliance_and_gradient(args, coords=None, include_surface=True):
    """Discrete compliance C = 1/2 U.F and dC/dP (3, nb_cp)."""
    coords = np.asarray(args[2] if coords is None else coords, dtype=np.float64)
    U, F = _solve(args, coords)
    a = list(args)
    a[2] = coords
    sol = U.reshape(-1, 3).T
    gi, ge = grad_from_system_args(a, sol, 0.5 * sol[None], True, True,
                                   include_surface)
    return 0.5 * U @ F, gi[0] + 2.0 * ge[0]


try:
    import torch

    class Compliance(torch.autograd.Function):
        """C(P) for control-point coordinates P (3, nb_cp) float64 tensor;
        ``Compliance.apply(P, args)`` with args the model's argument list of
        sys_linmat_lindef_static.  Backward: the adjoint kernel."""

        @staticmethod
        def forward(ctx, coords, args, include_surface=True):
            X = coords.detach().cpu().numpy()
            U, F = _solve(args, X)
            ctx.args = args
            ctx.X = X
            ctx.U = U
            ctx.include_surface = include_surface
            return torch.tensor(0.5 * U @ F, dtype=coords.dtype,
                                device=coords.device)

        @staticmethod
        def backward(ctx, grad_out):
            a = list(ctx.args)
            a[2] = ctx.X
            sol = ctx.U.reshape(-1, 3).T
            gi, ge = grad_from_system_args(a, sol, 0.5 * sol[None], True, True,
                                           ctx.include_surface)
            g = torch.from_numpy(gi[0] + 2.0 * ge[0]).to(grad_out.device)
            return grad_out * g.to(grad_out.dtype), None, None
except ImportError:   # torch is part of the runtime; keep the numpy API usable
    Compliance = None
