"""CPU oracle for the YETI U1 / weighted-quadrature / shape-gradient path.

TEST INFRASTRUCTURE ONLY: a restatement of the reference algorithm used to
check the CUDA product path.  Only tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` may import it.  The product package
(``yeti_b200``) never imports, links or calls anything under ``oracle/``.

The compiled part lives in ``yeti_oracle.c`` (assembly, plain C),
``oracle_wq.c`` and ``oracle_grad.c``; ``wq_rules.py`` / ``wq_ops.py`` hold the
numpy restatement of the weighted-quadrature rules and operator.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libyeti_oracle.so")
_lib = None


def build():
    """Compile the C oracle (``make -C oracle``)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
    return _lib


def threads():
    """OpenMP threads the oracle's element loops and WQ port use."""
    L = lib()
    L.oracle_wq_threads.restype = ctypes.c_int
    return int(L.oracle_wq_threads())


def _i64(a):
    return np.ascontiguousarray(np.asarray(a).ravel(order="F"), dtype=np.int64)


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _check_u1(elt_type, tensor, nb_patch):
    """The oracle restates the U1 / THREED branch only."""
    types = [t for t in str(elt_type).split("U")[1:]]
    if len(types) != nb_patch or any(t != "1" for t in types):
        raise NotImplementedError(f"oracle handles U1 patches only: {elt_type}")
    tens = [t for t in str(tensor).split("/") if t]
    if any(t != "THREED" for t in tens):
        raise NotImplementedError(f"oracle handles THREED only: {tensor}")


def sys_linmat_lindef_static(activeElement, nb_data, COORDS3D, IEN,
                             nb_elem_patch, Nkv, Ukv, Nijk, weight, Jpqr,
                             ELT_TYPE, PROPS, JPROPS, MATERIAL_PROPERTIES,
                             n_mat_props, RHO, TENSOR, indDLoad, JDLType,
                             ADLMAG, load_target_nbelem, load_additionalInfos,
                             nb_load_additionalInfos, bc_values, bc_target,
                             bc_target_nbelem, ind_dof_free, nb_dof_free,
                             MCRD, NBINT, NNODE, nodal_dist, nb_bc=None,
                             nb_load=None, nb_patch=None, nb_elem=None,
                             nb_cp=None, nb_dof_tot=None):
    """Oracle twin of ``stiffmtrx_elemstorage.sys_linmat_lindef_static``
    (``src/yeti_iga/main/build_system_elemStorage.f90:24-315``), same
    positional arguments as ``IGAparametrization.get_inputs4system_elemStorage``
    (``IGA_parametrization.py:1705-1716``).  Returns (Kdata, Krow, Kcol, F).
    """
    coords = np.asarray(COORDS3D, dtype=np.float64)
    nb_cp = coords.shape[1] if nb_cp is None else int(nb_cp)
    nb_patch = len(np.atleast_1d(nb_elem_patch)) if nb_patch is None else int(nb_patch)
    nb_elem = len(np.atleast_1d(activeElement)) if nb_elem is None else int(nb_elem)
    nb_dof_tot = int(MCRD) * nb_cp if nb_dof_tot is None else int(nb_dof_tot)
    if int(MCRD) != 3:
        raise NotImplementedError("oracle handles MCRD=3 only")
    _check_u1(ELT_TYPE, TENSOR, nb_patch)
    nb_data = int(nb_data)
    jdl = _i64(JDLType)
    nb_load = int(len(jdl)) if nb_load is None else int(nb_load)
    nodal = np.asarray(nodal_dist, dtype=np.float64)
    if nodal.ndim == 1:
        nodal = nodal.reshape(1, -1)
    nb_n_dist = nodal.shape[0]
    mat = np.asarray(MATERIAL_PROPERTIES, dtype=np.float64).reshape(-1, nb_patch, order="F")[:2]
    kdata = np.zeros(nb_data, dtype=np.float64)
    krow = np.zeros(nb_data, dtype=np.int32)
    kcol = np.zeros(nb_data, dtype=np.int32)
    F = np.zeros(nb_dof_tot, dtype=np.float64)
    keep = [_f64(coords), _i64(IEN), _i64(nb_elem_patch), _i64(Nkv), _f64(Ukv),
            _i64(Nijk), _f64(weight), _i64(Jpqr), _i64(NNODE), _i64(NBINT),
            _f64(mat), _f64(np.atleast_1d(RHO)), _i64(activeElement),
            _i64(indDLoad), jdl, _f64(ADLMAG), _i64(load_target_nbelem),
            _f64(load_additionalInfos), _i64(nb_load_additionalInfos),
            _f64(nodal)]
    f = lib().oracle_sys_linmat_lindef_static
    f.restype = ctypes.c_int
    i64 = ctypes.c_int64
    rc = f(i64(nb_patch), i64(nb_elem), i64(nb_cp), _p(keep[0]), _p(keep[1]),
           _p(keep[2]), _p(keep[3]), _p(keep[4]), _p(keep[5]), _p(keep[6]),
           _p(keep[7]), _p(keep[8]), _p(keep[9]), _p(keep[10]), _p(keep[11]),
           _p(keep[12]), i64(nb_load), _p(keep[13]), _p(keep[14]),
           _p(keep[15]), _p(keep[16]), _p(keep[17]), _p(keep[18]),
           i64(nb_n_dist), _p(keep[19]), i64(nb_data), i64(nb_dof_tot),
           _p(kdata), _p(krow), _p(kcol), _p(F))
    if rc != 0:
        raise RuntimeError(f"oracle assembly failed with code {rc}")
    return kdata, krow, kcol, F


def grad_lin_elast_work(args, sol, adj, compute_int=True, compute_ext=True,
                        include_surface=False):
    """Oracle twin of gradadjointwork.gradlinelastwork_an
    (src/yeti_iga/optim/gradtotalwork_fullAN.f90:17-300) for U1 patches.

    args: the positional list of get_inputs4system_elemStorage (the model);
    sol: (3, nb_cp); adj: (nadj, 3, nb_cp).  Returns (gradWint, gradWext),
    each (nadj, 3, nb_cp).  include_surface adds the surface-load sensitivity
    the reference leaves out (gradUELMAT_solid.f90:463-477)."""
    (activeElement, nb_data, COORDS3D, IEN, nb_elem_patch, Nkv, Ukv, Nijk,
     weight, Jpqr, ELT_TYPE, PROPS, JPROPS, MATERIAL_PROPERTIES, n_mat_props,
     RHO, TENSOR, indDLoad, JDLType, ADLMAG, load_target_nbelem,
     load_additionalInfos, nb_load_additionalInfos, bc_values, bc_target,
     bc_target_nbelem, ind_dof_free, nb_dof_free, MCRD, NBINT, NNODE,
     nodal_dist) = args[:32]
    coords = np.asarray(COORDS3D, dtype=np.float64)
    nb_cp = coords.shape[1]
    nb_patch = len(np.atleast_1d(nb_elem_patch))
    _check_u1(ELT_TYPE, TENSOR, nb_patch)
    adj = np.asarray(adj, dtype=np.float64)
    nadj = adj.shape[0]
    nodal = np.asarray(nodal_dist, dtype=np.float64)
    if nodal.ndim == 1:
        nodal = nodal.reshape(1, -1)
    mat = np.asarray(MATERIAL_PROPERTIES, dtype=np.float64).reshape(-1, nb_patch, order="F")[:2]
    jdl = _i64(JDLType)
    keep = [_f64(coords), _i64(IEN), _i64(nb_elem_patch), _i64(Nkv), _f64(Ukv),
            _i64(Nijk), _f64(weight), _i64(Jpqr), _i64(NNODE), _i64(NBINT),
            _f64(mat), _f64(np.atleast_1d(RHO)), _i64(activeElement),
            _i64(indDLoad), jdl, _f64(ADLMAG), _i64(load_target_nbelem),
            _f64(load_additionalInfos), _f64(nodal), _f64(sol), _f64(adj)]
    gi = np.zeros((nadj, 3, nb_cp), order="F")
    ge = np.zeros((nadj, 3, nb_cp), order="F")
    f = lib().oracle_grad_lin_elast_work
    f.restype = ctypes.c_int
    i64 = ctypes.c_int64
    rc = f(i64(nb_patch), i64(len(keep[12])), i64(nb_cp), _p(keep[0]), _p(keep[1]),
           _p(keep[2]), _p(keep[3]), _p(keep[4]), _p(keep[5]), _p(keep[6]),
           _p(keep[7]), _p(keep[8]), _p(keep[9]), _p(keep[10]), _p(keep[11]),
           _p(keep[12]), i64(len(jdl)), _p(keep[13]), _p(keep[14]), _p(keep[15]),
           _p(keep[16]), _p(keep[17]), i64(nodal.shape[0]), _p(keep[18]),
           _p(keep[19]), _p(keep[20]), i64(nadj), ctypes.c_int(int(compute_int)),
           ctypes.c_int(int(compute_ext)), ctypes.c_int(int(include_surface)),
           gi.ctypes.data_as(ctypes.c_void_p), ge.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise RuntimeError(f"oracle gradient failed with code {rc}")
    return gi, ge


def volume(area_inputs, gradient=True):
    """Oracle twin of volume.computevolume / computegradvolume
    (src/yeti_iga/optim/volume.f90:20-210, gradvolume.f90:16-355) for U1
    patches.  area_inputs: the list of IGAparametrization.get_inputs4area.
    Returns (V, dV/dP of shape (3, nb_cp) or None)."""
    (listpatch, COORDS3D, IEN, nb_elem_patch, Nkv, Ukv, Nijk, weight, Jpqr,
     ELT_TYPE, PROPS, JPROPS, TENSOR, MCRD, NBINT, nnode) = area_inputs[:16]
    coords = np.asarray(COORDS3D, dtype=np.float64)
    nb_cp = coords.shape[1]
    nep = _i64(nb_elem_patch)
    _check_u1(ELT_TYPE, TENSOR, nep.size)
    keep = [_f64(coords), _i64(IEN), nep, _i64(Nkv), _f64(Ukv), _i64(Nijk),
            _f64(weight), _i64(Jpqr), _i64(nnode), _i64(NBINT), _i64(listpatch)]
    vol = ctypes.c_double()
    grad = np.zeros((3, nb_cp), order="F") if gradient else None
    f = lib().oracle_volume
    f.restype = ctypes.c_int
    rc = f(ctypes.c_int64(nep.size), ctypes.c_int64(nb_cp), *[_p(k) for k in keep],
           ctypes.byref(vol), _p(grad) if gradient else None)
    if rc != 0:
        raise RuntimeError(f"oracle_volume failed ({rc})")
    return vol.value, grad


def build_cmassmatrix(inputs):
    """Oracle twin of massmtrx.build_cmassmatrix (compute_CMASSMatrix.f:30-199,
    UMASSMAT.f U1 branch).  inputs: the list of
    IGAparametrization.get_inputs4massmat.  Returns (Mdata, Mrow, Mcol)."""
    (activeElement, nb_data, COORDS3D, IEN, nb_elem_patch, Nkv, Ukv, Nijk, weight,
     Jpqr, ELT_TYPE, PROPS, JPROPS, RHO, TENSOR, ind_dof_free, nb_dof_free, MCRD,
     NBINT, nnode) = inputs[:20]
    coords = np.asarray(COORDS3D, dtype=np.float64)
    nep = _i64(nb_elem_patch)
    _check_u1(ELT_TYPE, TENSOR, nep.size)
    act = _i64(activeElement)
    keep = [_f64(coords), _i64(IEN), nep, _i64(Nkv), _f64(Ukv), _i64(Nijk), _f64(weight),
            _i64(Jpqr), _i64(nnode), _i64(NBINT), _f64(np.atleast_1d(RHO)), act]
    n = int(nb_data)
    md, mr, mc = np.empty(n), np.empty(n, dtype=np.int32), np.empty(n, dtype=np.int32)
    f = lib().oracle_build_cmassmatrix
    f.restype = ctypes.c_int
    i64 = ctypes.c_int64
    rc = f(i64(nep.size), i64(act.size), i64(coords.shape[1]), *[_p(k) for k in keep],
           i64(n), _p(md), _p(mr), _p(mc))
    if rc != 0:
        raise RuntimeError(f"oracle_build_cmassmatrix failed ({rc})")
    return md, mr, mc
