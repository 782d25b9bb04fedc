"""Drop-in for the reference's ``yeti_iga.stiffmtrx_elemstorage`` f2py module.

``sys_linmat_lindef_static(*IGAparametrization.get_inputs4system_elemStorage())``
returns ``(Kdata, Krow, Kcol, F)`` exactly like the Fortran routine
(``src/yeti_iga/main/build_system_elemStorage.f90:24-315``): the
upper-triangle 3x3 blocks of every active U1 element in COO form (diagonal
blocks halved, so ``K = Kside + Kside.T``), 0-based int32 row/column dof
indices, and the load vector.  The work runs on the GPU through
``yeti_assemble_u1_coo`` in libyeti_b200.so; there is no CPU path.
"""
import numpy as np

from . import _lib
from ._lib import MEM_DEVICE, MEM_HOST, U1Model, check, lib, ptr

__all__ = ["sys_linmat_lindef_static", "pack_u1_model", "SYSTEM_ARG_NAMES"]

# The 38 positional arguments, in the order of
# IGAparametrization.get_inputs4system_elemStorage()
# (IGA_parametrization.py:1705-1716).
SYSTEM_ARG_NAMES = [
    "activeElement", "nb_data", "COORDS3D", "IEN", "nb_elem_patch", "Nkv",
    "Ukv", "Nijk", "weight", "Jpqr", "ELT_TYPE", "PROPS", "JPROPS",
    "MATERIAL_PROPERTIES", "n_mat_props", "RHO", "TENSOR", "indDLoad",
    "JDLType", "ADLMAG", "load_target_nbelem", "load_additionalInfos",
    "nb_load_additionalInfos", "bc_values", "bc_target", "bc_target_nbelem",
    "ind_dof_free", "nb_dof_free", "MCRD", "NBINT", "NNODE", "nodal_dist",
    "nb_bc", "nb_load", "nb_patch", "nb_elem", "nb_cp", "nb_dof_tot",
]


def _i64(a):
    return np.ascontiguousarray(np.asarray(a).ravel(order="F"), dtype=np.int64)


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))


def _split_elt_types(elt_type, nb_patch):
    s = str(elt_type)
    types = ["U" + t for t in s.split("U")[1:]]
    if len(types) != nb_patch:
        raise ValueError(f"ELT_TYPE {s!r} does not name {nb_patch} patches")
    return types


def _split_tensor(tensor, nb_patch):
    parts = [t for t in str(tensor).split("/")[1:]]
    if len(parts) != nb_patch:
        raise ValueError(f"TENSOR {tensor!r} does not name {nb_patch} patches")
    return parts


class PackedModel:
    """A yeti_u1_model plus the numpy arrays its pointers refer to."""

    def __init__(self, arrays, struct, nb_data, nb_dof_tot):
        self.arrays = arrays
        self.struct = struct
        self.nb_data = nb_data
        self.nb_dof_tot = nb_dof_tot


def pack_u1_model(activeElement, nb_data, COORDS3D, IEN, nb_elem_patch, Nkv,
                  Ukv, Nijk, weight, Jpqr, ELT_TYPE, PROPS, JPROPS,
                  MATERIAL_PROPERTIES, n_mat_props, RHO, TENSOR, indDLoad,
                  JDLType, ADLMAG, load_target_nbelem, load_additionalInfos,
                  nb_load_additionalInfos, bc_values, bc_target,
                  bc_target_nbelem, ind_dof_free, nb_dof_free, MCRD, NBINT,
                  NNODE, nodal_dist, nb_bc=None, nb_load=None, nb_patch=None,
                  nb_elem=None, nb_cp=None, nb_dof_tot=None):
    """Convert the reference's positional argument list into a yeti_u1_model."""
    if int(MCRD) != 3:
        raise NotImplementedError("only 3D (MCRD=3) solids are on this path")
    coords = np.asarray(COORDS3D, dtype=np.float64)
    if coords.ndim != 2 or coords.shape[0] != 3:
        raise ValueError("COORDS3D must have shape (3, nb_cp)")
    nb_cp = coords.shape[1] if nb_cp is None else int(nb_cp)
    nep = _i64(nb_elem_patch)
    nb_patch = nep.size if nb_patch is None else int(nb_patch)
    act = _i64(activeElement)
    nb_elem = act.size if nb_elem is None else int(nb_elem)
    nb_dof_tot = 3 * nb_cp if nb_dof_tot is None else int(nb_dof_tot)
    types = _split_elt_types(ELT_TYPE, nb_patch)
    tens = _split_tensor(TENSOR, nb_patch)
    is_u1 = np.array([1 if (t == "U1" and tt == "THREED") else 0
                      for t, tt in zip(types, tens)], dtype=np.int32)
    mat = np.asarray(MATERIAL_PROPERTIES, dtype=np.float64)
    mat = mat.reshape(-1, nb_patch, order="F")[:2]
    jdl = _i64(JDLType)
    nb_load = jdl.size if nb_load is None else int(nb_load)
    nodal = np.asarray(nodal_dist, dtype=np.float64)
    if nodal.ndim == 1:
        nodal = nodal.reshape(1, -1)
    infos = _f64(load_additionalInfos)
    arrays = dict(
        coords=_f64(coords), ien=_i64(IEN), nb_elem_patch=nep, nkv=_i64(Nkv),
        ukv=_f64(Ukv), nijk=_i64(Nijk), weight=_f64(weight), jpqr=_i64(Jpqr),
        nnode=_i64(NNODE), nbint=_i64(NBINT), is_u1=is_u1, matprops=_f64(mat),
        rho=_f64(np.atleast_1d(RHO)), active=act, inddload=_i64(indDLoad),
        jdltype=jdl, adlmag=_f64(ADLMAG),
        load_target_nbelem=_i64(load_target_nbelem), load_addinfos=infos,
        nb_load_addinfos=_i64(nb_load_additionalInfos), nodal_dist=_f64(nodal))
    if arrays["nb_load_addinfos"].size < nb_load:
        arrays["nb_load_addinfos"] = np.zeros(max(nb_load, 1), dtype=np.int64)
    s = U1Model()
    s.nb_patch, s.nb_elem, s.nb_cp = nb_patch, nb_elem, nb_cp
    for k in ("coords", "ien", "nb_elem_patch", "nkv", "ukv", "nijk", "weight",
              "jpqr", "nnode", "nbint", "is_u1", "matprops", "rho", "active",
              "inddload", "jdltype", "adlmag", "load_target_nbelem",
              "load_addinfos", "nb_load_addinfos", "nodal_dist"):
        setattr(s, k, arrays[k].ctypes.data)
    s.nb_load = nb_load
    s.len_load_addinfos = infos.size
    s.nb_n_dist = nodal.shape[0]
    return PackedModel(arrays, s, int(nb_data), nb_dof_tot)


def sys_linmat_lindef_static(*args, ctx=None, device_out=False,
                             element_kernel="pairs", **kwargs):
    """GPU twin of ``stiffmtrx_elemstorage.sys_linmat_lindef_static``.

    Positional arguments: the 38 items of
    ``IGAparametrization.get_inputs4system_elemStorage()``
    (``IGA_parametrization.py:1705-1716``).  Returns numpy
    ``(Kdata float64, Krow int32, Kcol int32, F float64)``; with
    ``device_out=True`` the four are torch CUDA tensors instead.

    ``element_kernel``: ``"pairs"`` (default) sums each control-point pair's
    block over the Gauss points in the reference's operation order, so the
    values are bit-identical to it; ``"sumfact"`` contracts BᵀDB direction by
    direction over the 1-D basis tables (same slots, values equal to
    rounding, far fewer operations from degree 3 on).
    """
    kinds = {"pairs": _lib.STIFF_PAIRS, "sumfact": _lib.STIFF_SUMFACT}
    if element_kernel not in kinds:
        raise ValueError(f"element_kernel must be one of {sorted(kinds)}")
    pm = pack_u1_model(*args, **kwargs)
    ctx = ctx or _lib.default_context()
    n = pm.nb_data
    if device_out:
        import torch
        dev = torch.device("cuda", ctx.device)
        kdata = torch.empty(n, dtype=torch.float64, device=dev)
        krow = torch.empty(n, dtype=torch.int32, device=dev)
        kcol = torch.empty(n, dtype=torch.int32, device=dev)
        F = torch.empty(pm.nb_dof_tot, dtype=torch.float64, device=dev)
        mem = MEM_DEVICE
    else:
        kdata = np.empty(n, dtype=np.float64)
        krow = np.empty(n, dtype=np.int32)
        kcol = np.empty(n, dtype=np.int32)
        F = np.empty(pm.nb_dof_tot, dtype=np.float64)
        mem = MEM_HOST
    check(lib().yeti_assemble_u1_coo_ex(ctx.handle, pm.struct, n, ptr(kdata),
                                        ptr(krow), ptr(kcol), ptr(F), mem,
                                        kinds[element_kernel]),
          "yeti_assemble_u1_coo")
    return kdata, krow, kcol, F
