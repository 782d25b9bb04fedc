"""Generate the model-array fixtures under tests/golden/ from the reference's
own Python preprocessing.

The reference (arnaudduval/yeti) reads Abaqus-like ``.inp`` + ``.NB`` model
files and k-refines them in pure Python
(``preprocessing/igaparametrization/IGA_parametrization.py`` and
``IGA_refinementFcts.py``).  Its compiled Fortran extension modules cannot be
built in this environment (no Fortran compiler), so they are replaced by stubs
here; the only one whose *result* is used, ``DOF.getinddof``, is restated in
numpy below from ``src/yeti_iga/main/indDOF.f:18-110``.

The script runs where the reference source tree is available (set
``YETI_REFERENCE`` to its root).  It writes ``tests/golden/*.npz``: exactly the
positional argument list that ``IGAparametrization.get_inputs4system_elemStorage``
(``IGA_parametrization.py:1659-1718``) hands to
``stiffmtrx_elemstorage.sys_linmat_lindef_static``, plus the data the known-answer
checks of the reference's own tests need.  Nothing at test time imports the
reference: the tests read these files.

Usage:  python tests/golden/make_fixtures.py
"""
import importlib
import importlib.machinery
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("YETI_REFERENCE", "")
MODELS = os.path.join(HERE, "models")


# ---------------------------------------------------------------------------
# stubs for the compiled (f2py) modules of the reference
# ---------------------------------------------------------------------------
def _getinddof(mcrd, bc_target, bc_target_nbelem, bc_values, nb_dof_tot,
               nb_bc, bc_target_size):
    """numpy restatement of getindDOF (``src/yeti_iga/main/indDOF.f:18-110``).

    Returns (nb_dof_bloq, nb_dof_free, ind_dof_bloq, ind_dof_free,
    COUPLG_flag, BNDSTRIP_flag) with 1-based dof indices, zero padded to
    nb_dof_tot like the Fortran output arrays.
    """
    test = np.zeros(nb_dof_tot, dtype=np.int64)
    couplg = False
    bndstrip = False
    count = 0
    bc_values = np.asarray(bc_values, dtype=np.float64).reshape(2, -1)
    bc_target = np.asarray(bc_target).ravel()
    for ibc in range(int(nb_bc)):
        n = int(bc_target_nbelem[ibc])
        code = bc_values[0, ibc]
        cps = bc_target[count:count + n]
        if code == 11.0:
            bndstrip = True
        elif code == 10.0:
            couplg = True
            for cp in cps:
                ddl = (int(cp) - 1) * mcrd
                test[ddl:ddl + 3] = 1
        else:
            direction = int(code)
            if 6.0 < code < 10.0:
                direction -= 6
                couplg = True
            for cp in cps:
                test[(int(cp) - 1) * mcrd + direction - 1] = 1
        count += n
    bloq = np.nonzero(test == 1)[0] + 1
    free = np.nonzero(test == 0)[0] + 1
    ind_bloq = np.zeros(nb_dof_tot, dtype=np.int64)
    ind_free = np.zeros(nb_dof_tot, dtype=np.int64)
    ind_bloq[:bloq.size] = bloq
    ind_free[:free.size] = free
    return bloq.size, free.size, ind_bloq, ind_free, couplg, bndstrip


def _install_stubs():
    pkg_dir = os.path.join(REF, "src", "yeti_iga")
    if not REF or not os.path.isdir(pkg_dir):
        raise SystemExit("set YETI_REFERENCE to the root of the reference source tree")

    def mod(name, **attrs):
        m = types.ModuleType(name)
        for k, v in attrs.items():
            setattr(m, k, v)
        sys.modules[name] = m
        return m

    def unavailable(*_a, **_k):
        raise RuntimeError("compiled reference module is stubbed here")

    # The package itself: skip its __init__ (it pulls every f2py module).
    root = mod("yeti_iga")
    root.__path__ = [pkg_dir]
    mod("yeti_iga.DOF", getinddof=_getinddof)

    class _StubFinder:
        """Serve a stub for every yeti_iga submodule that has no Python
        source (those are the f2py-compiled extensions)."""

        def find_spec(self, name, path=None, target=None):
            if not name.startswith("yeti_iga."):
                return None
            rel = os.path.join(pkg_dir, *name.split(".")[1:])
            if os.path.isdir(rel) or os.path.isfile(rel + ".py"):
                return None
            return importlib.machinery.ModuleSpec(name, self)

        def create_module(self, spec):
            m = types.ModuleType(spec.name)
            m.__getattr__ = lambda attr: unavailable
            return m

        def exec_module(self, module):
            pass

    sys.meta_path.append(_StubFinder())
    for sub in ("postprocessing", "fitting", "coupling", "optim", "solver"):
        d = os.path.join(pkg_dir, sub)
        if os.path.isdir(d) and os.path.isfile(os.path.join(d, "__init__.py")):
            continue
        p = mod("yeti_iga." + sub)
        p.__path__ = [d]


def _load_igaparam():
    _install_stubs()
    m = importlib.import_module(
        "yeti_iga.preprocessing.igaparametrization.IGA_parametrization")
    return m.IGAparametrization


# ---------------------------------------------------------------------------
# fixture writers
# ---------------------------------------------------------------------------
SYSTEM_ARG_NAMES = [
    "activeElement", "nb_data", "COORDS3D", "IEN", "nb_elem_patch", "Nkv",
    "Ukv", "Nijk", "weight", "Jpqr", "ELT_TYPE", "PROPS", "JPROPS",
    "MATERIAL_PROPERTIES", "n_mat_props", "RHO", "TENSOR", "indDLoad",
    "JDLType", "ADLMAG", "load_target_nbelem", "load_additionalInfos",
    "nb_load_additionalInfos", "bc_values", "bc_target", "bc_target_nbelem",
    "ind_dof_free", "nb_dof_free", "MCRD", "NBINT", "NNODE", "nodal_dist",
    "nb_bc", "nb_load", "nb_patch", "nb_elem", "nb_cp", "nb_dof_tot",
]


def _save_model(name, igap, extra=None):
    args = igap.get_inputs4system_elemStorage()
    assert len(args) == len(SYSTEM_ARG_NAMES), len(args)
    out = {}
    for key, val in zip(SYSTEM_ARG_NAMES, args):
        if isinstance(val, str):
            out[key] = np.array(val)
        else:
            arr = np.asarray(val)
            if arr.dtype == object:
                arr = arr.astype(np.float64)
            out[key] = arr
    if extra:
        out.update(extra)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: nb_elem={int(out['nb_elem'])} "
          f"nb_cp={int(out['nb_cp'])} nb_data={int(out['nb_data'])}")


def main():
    IGAparametrization = _load_igaparam()
    # the .inp reader writes <part>.save files into the working directory
    import tempfile
    os.chdir(tempfile.mkdtemp(prefix="yeti_fixtures_"))

    # 1. benchs/omp/test_build_stifmatrix_omp.py:41-73 model
    m = IGAparametrization(filename=os.path.join(REF, "benchs/omp/beam-dist"))
    m.refine(np.array([2, 2, 2]), np.array([2, 2, 2]))
    _save_model("omp_beam_dist", m)

    # 2. benchs/dload/test_dload_beam_dist.py:39-81 (deflection -1142.857,
    #    rtol 2e-2, z displacement of the control point at (20, 0, 0))
    m = IGAparametrization(filename=os.path.join(REF, "benchs/dload/beam-dist"))
    m.refine(np.array([2, 2, 5]), np.array([1, 1, 1]))
    coords = np.asarray(m.coords)
    idx = int(np.nonzero(np.all(coords.T == [20.0, 0.0, 0.0], axis=1))[0][0])
    _save_model("dload_beam_dist", m, {
        "check_cp": np.array(idx), "check_comp": np.array(2),
        "check_value": np.array(-1142.857), "check_rtol": np.array(2e-2)})

    # 3. benchs/volume_force/test_volume_force_3d.py:41-80 (displacement at
    #    xi=(1,1,0) vs Abaqus, relative error < 2e-3).  xi=(1,1,0) is a patch
    #    corner, where an open-knot NURBS patch interpolates its corner CP.
    m = IGAparametrization(
        filename=os.path.join(REF, "benchs/volume_force/volume_force_3D"))
    nb_deg = np.zeros((3, m.nb_patch), dtype=np.intp)
    nb_ref = np.zeros((3, m.nb_patch), dtype=np.intp)
    nb_deg[:, 0] = [1, 1, 1]
    nb_ref[:, 0] = [3, 4, 3]
    m.refine(nb_ref, nb_deg)
    ind = m._indCPbyPatch[0] - 1
    nkv = np.asarray(m._Nkv)[:, 0]
    jpqr = np.asarray(m._Jpqr)[:, 0]
    ncp = nkv - jpqr - 1
    corner = int(ind[(ncp[0] - 1) + (ncp[1] - 1) * ncp[0]])
    _save_model("volume_force_3d", m, {
        "check_cp": np.array(corner),
        "check_disp": np.array([-9.96639E-5, -1.01212, -6.42538]),
        "check_rtol": np.array(2e-3)})

    # 4. cantilever block 10x1x1, p=2, 16x4x4 elements, E=210000, nu=0.3,
    #    clamped at x=0, traction 1.0 in -z on the x=10 face
    m = IGAparametrization(filename=os.path.join(MODELS, "cantilever_block"))
    m.refine(np.array([4, 2, 2]), np.array([1, 1, 1]))
    _save_model("cantilever_p2_16x4x4", m)

    # 5. benchs/grad_solid/test_grad_solid_unit_cube_centrif.py model
    #    (p=1 unit cube, centrifugal body load U101)
    m = IGAparametrization(
        filename=os.path.join(REF, "benchs/grad_solid/unit_cube_U1"))
    _save_model("grad_unit_cube", m)

    # 6. quarter annulus (R 1 -> 4, thickness 0.1), exact circular arcs,
    #    p=2 everywhere, 32x32x2 elements, outward radial pressure on the
    #    outer face, symmetry on the straight faces, u_z = 0 on z = 0
    m = IGAparametrization(filename=os.path.join(MODELS, "quarter_annulus"))
    m.refine(np.array([5, 5, 1]), np.array([1, 0, 1]))
    _save_model("quarter_annulus_p2_32x32x2", m)
    m = IGAparametrization(filename=os.path.join(MODELS, "quarter_annulus"))
    m.refine(np.array([2, 2, 1]), np.array([1, 0, 1]))
    _save_model("quarter_annulus_p2_4x4x2", m)


if __name__ == "__main__":
    main()
