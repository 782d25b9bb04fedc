"""Volume of U1 solid patches and its shape gradient on the GPU.

``computevolume`` / ``computegradvolume`` are the drop-ins for the
reference's ``optim.volume.computevolume`` / ``computegradvolume``
(``src/yeti_iga/optim/volume.f90:20-210``, ``gradvolume.f90:16-355``), called
by ``OPTmodelling.compute_volume`` / ``compute_gradVolume_AN``
(``preprocessing/igaparametrization/OPT_modelling.py:508-531``) with the list
of ``IGAparametrization.get_inputs4area`` (``IGA_parametrization.py:
1286-1312``).  Both run ``yeti_volume_u1`` in libyeti_b200.so.

``Volume`` is a ``torch.autograd.Function``: V(P) for control-point
coordinates P (3, nb_cp), backward dV/dP, for a volume constraint beside the
compliance of ``yeti_b200.gradient.Compliance``.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import MEM_HOST, check, lib, ptr
from .stiffmtrx_elemstorage import pack_u1_model

__all__ = ["computevolume", "computegradvolume", "volume_and_gradient", "Volume"]


def _pack_area(listpatch, COORDS3D, IEN, nb_elem_patch, Nkv, Ukv, Nijk, weight,
               Jpqr, ELT_TYPE, PROPS, JPROPS, TENSOR, MCRD, NBINT, nnode,
               nb_patch=None, nb_elem=None, nb_cp=None):
    """The get_inputs4area list as a yeti_u1_model: listpatch selects whole
    patches (every element of a listed patch is active)."""
    nep = np.atleast_1d(np.asarray(nb_elem_patch, dtype=np.int64))
    npatch = nep.size
    lp = np.atleast_1d(np.asarray(listpatch, dtype=np.int64))
    if lp.size != npatch:
        raise ValueError(f"listpatch has {lp.size} entries for {npatch} patches")
    coords = np.asarray(COORDS3D, dtype=np.float64)
    active = np.repeat((lp == 1).astype(np.int64), nep)
    no_i, no_f = np.zeros(1, dtype=np.int64), np.zeros(1)
    args = [active, 0, coords, IEN, nep, Nkv, Ukv, Nijk, weight, Jpqr,
            ELT_TYPE, PROPS, JPROPS, np.ones((2, npatch)), 2, np.zeros(npatch),
            TENSOR, no_i, np.zeros(0, dtype=np.int64), np.zeros(0),
            np.zeros(0, dtype=np.int64), no_f, no_i, no_f, no_i, no_i, no_i, 0,
            MCRD, NBINT, nnode, np.zeros((1, coords.shape[1]))]
    return pack_u1_model(*args)


def volume_and_gradient(area_inputs, gradient=True, ctx=None):
    """(V, dV/dP (3, nb_cp) or None) for the get_inputs4area list."""
    pm = _pack_area(*area_inputs)
    ctx = ctx or _lib.default_context()
    vol = ctypes.c_double()
    grad = np.zeros((3, pm.struct.nb_cp), order="F") if gradient else None
    check(lib().yeti_volume_u1(ctx.handle, ctypes.byref(pm.struct), ctypes.byref(vol),
                               ptr(grad) if gradient else None, MEM_HOST),
          "yeti_volume_u1")
    return vol.value, grad


def computevolume(*area_inputs, ctx=None):
    """GPU twin of volume.computevolume: the volume of the listed patches."""
    return volume_and_gradient(area_inputs, gradient=False, ctx=ctx)[0]


def computegradvolume(*area_inputs, ctx=None):
    """GPU twin of volume.computegradvolume: dV/dP, shape (3, nb_cp)."""
    return volume_and_gradient(area_inputs, gradient=True, ctx=ctx)[1]


try:
    import torch

    class Volume(torch.autograd.Function):
        """V(P) for control-point coordinates P (3, nb_cp) float64 tensor;
        ``Volume.apply(P, area_inputs)`` with area_inputs the
        get_inputs4area list (its coordinates are replaced by P)."""

        @staticmethod
        def forward(ctx, coords, area_inputs):
            a = list(area_inputs)
            a[1] = coords.detach().cpu().numpy()
            v, g = volume_and_gradient(a, gradient=True)
            ctx.g = g
            return torch.tensor(v, dtype=coords.dtype, device=coords.device)

        @staticmethod
        def backward(ctx, grad_out):
            g = torch.from_numpy(np.ascontiguousarray(ctx.g)).to(grad_out.device)
            return grad_out * g.to(grad_out.dtype), None
except ImportError:   # torch is part of the runtime; keep the numpy API usable
    Volume = None
