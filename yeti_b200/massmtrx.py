"""Consistent mass matrix of U1 solids on the GPU.

``build_cmassmatrix`` is the drop-in for the reference's
``massmtrx.build_cmassmatrix`` (``build_CMASSMatrix``,
``src/yeti_iga/main/compute_CMASSMatrix.f:30-199``, with ``UMASSMAT_byCP``,
``main/UMASSMAT.f``), called at
``preprocessing/igaparametrization/OPT_modelling.py:369-371`` with the list of
``IGAparametrization.get_inputs4massmat`` (``IGA_parametrization.py:
1720-1764``).  It runs ``yeti_assemble_u1_mass_coo`` in libyeti_b200.so and
returns ``(Mdata, Mrow, Mcol)`` in the stiffness assembly's COO slot order
(upper-triangle blocks, diagonal of the diagonal blocks halved): the caller
forms ``M = Mside + Mside.T`` as for the stiffness.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import MEM_DEVICE, MEM_HOST, check, lib, ptr
from .stiffmtrx_elemstorage import pack_u1_model

__all__ = ["build_cmassmatrix"]


def build_cmassmatrix(activeElement, nb_data, COORDS3D, IEN, nb_elem_patch, Nkv,
                      Ukv, Nijk, weight, Jpqr, ELT_TYPE, PROPS, JPROPS, RHO,
                      TENSOR, ind_dof_free, nb_dof_free, MCRD, NBINT, nnode,
                      nb_patch=None, nb_elem=None, nb_cp=None, nb_dof_tot=None,
                      ctx=None, device_out=False):
    """GPU twin of massmtrx.build_cmassmatrix (same positional arguments).
    Returns (Mdata, Mrow, Mcol) as numpy arrays, or torch CUDA tensors with
    device_out=True."""
    nep = np.atleast_1d(np.asarray(nb_elem_patch, dtype=np.int64))
    npatch = nep.size
    coords = np.asarray(COORDS3D, dtype=np.float64)
    no_i, no_f = np.zeros(1, dtype=np.int64), np.zeros(1)
    args = [activeElement, nb_data, coords, IEN, nep, Nkv, Ukv, Nijk, weight, Jpqr,
            ELT_TYPE, PROPS, JPROPS, np.ones((2, npatch)), 2,
            np.atleast_1d(np.asarray(RHO, dtype=np.float64)), TENSOR, no_i,
            np.zeros(0, dtype=np.int64), np.zeros(0), np.zeros(0, dtype=np.int64), no_f,
            no_i, no_f, no_i, no_i, no_i, 0, MCRD, NBINT, nnode,
            np.zeros((1, coords.shape[1]))]
    pm = pack_u1_model(*args)
    ctx = ctx or _lib.default_context()
    n = int(nb_data)
    if device_out:
        import torch
        dev = torch.device("cuda", ctx.device)
        md = torch.empty(n, dtype=torch.float64, device=dev)
        mr = torch.empty(n, dtype=torch.int32, device=dev)
        mc = torch.empty(n, dtype=torch.int32, device=dev)
        mem = MEM_DEVICE
    else:
        md, mr, mc = np.empty(n), np.empty(n, dtype=np.int32), np.empty(n, dtype=np.int32)
        mem = MEM_HOST
    check(lib().yeti_assemble_u1_mass_coo(ctx.handle, ctypes.byref(pm.struct), n, ptr(md),
                                          ptr(mr), ptr(mc), mem),
          "yeti_assemble_u1_mass_coo")
    return md, mr, mc
