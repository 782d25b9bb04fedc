"""U1 element stiffness + COO assembly: oracle pins (CPU) and GPU parity.

Parity bar (the reference's own seq-vs-OpenMP test style,
benchs/omp/test_build_stifmatrix_omp.py:41-73): identical Krow/Kcol,
||dKdata||/||Kdata|| <= 1e-12 and max|dKdata| <= 1e-12 max|Kdata|,
||dF||/||F|| <= 1e-12, and the direct-solve displacement within 1e-12.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle
from conftest import load_fixture

FIXTURES = ["cantilever_p2_16x4x4", "dload_beam_dist", "volume_force_3d",
            "omp_beam_dist", "grad_unit_cube", "quarter_annulus_p2_4x4x2"]
TOL = 1e-12


def _solve(d, kdata, krow, kcol, rhs):
    ndof = int(d["nb_dof_tot"])
    K = sp.coo_matrix((kdata, (krow, kcol)), shape=(ndof, ndof)).tocsc()
    K = K + K.T
    idof = d["ind_dof_free"][:int(d["nb_dof_free"])] - 1
    x = spla.spsolve(K[idof, :][:, idof], rhs[idof])
    sol = np.zeros(ndof)
    sol[idof] = x
    return sol.reshape(-1, 3)


# ----------------------------------------------------------------- CPU: oracle
def test_oracle_dload_beam_known_answer():
    """benchs/dload/test_dload_beam_dist.py:66-81: tip deflection -1142.857
    (analytic), rtol 2e-2, for the p=2 refined beam under normal pressure."""
    d, args = load_fixture("dload_beam_dist")
    sol = _solve(d, *oracle.sys_linmat_lindef_static(*args))
    val = sol[int(d["check_cp"]), int(d["check_comp"])]
    assert np.isclose(val, float(d["check_value"]), rtol=float(d["check_rtol"]))


def test_oracle_volume_force_known_answer():
    """benchs/volume_force/test_volume_force_3d.py:38,74-80: Abaqus
    displacement at xi=(1,1,0), relative error < 2e-3 (U102 body force)."""
    d, args = load_fixture("volume_force_3d")
    sol = _solve(d, *oracle.sys_linmat_lindef_static(*args))
    v = sol[int(d["check_cp"])]
    ref = d["check_disp"]
    assert np.linalg.norm(v - ref) / np.linalg.norm(ref) < float(d["check_rtol"])


def test_oracle_cantilever_resultant_and_beam_theory():
    """Cantilever 10x1x1 (E=210000): the traction resultant is exactly -1 in z
    and the tip deflection is close to Euler-Bernoulli P L^3 / (3 E I)."""
    d, args = load_fixture("cantilever_p2_16x4x4")
    kdata, krow, kcol, F = oracle.sys_linmat_lindef_static(*args)
    assert int(d["nb_data"]) == 850176
    Fz = F.reshape(-1, 3)
    assert np.isclose(Fz[:, 2].sum(), -1.0, rtol=1e-13)
    assert np.abs(Fz[:, :2]).max() == 0.0
    sol = _solve(d, kdata, krow, kcol, F)
    eb = 1.0 * 10.0 ** 3 / (3 * 210000.0 * (1.0 / 12.0))
    assert np.isclose(sol[:, 2].min(), -eb, rtol=0.05)


def test_oracle_stiffness_is_symmetric_psd_with_rigid_modes():
    """K = Kside + Kside^T annihilates the 6 rigid-body modes of the
    unconstrained single-element cube."""
    d, args = load_fixture("grad_unit_cube")
    kdata, krow, kcol, _ = oracle.sys_linmat_lindef_static(*args)
    n = int(d["nb_dof_tot"])
    K = sp.coo_matrix((kdata, (krow, kcol)), shape=(n, n)).toarray()
    K = K + K.T
    X = d["COORDS3D"].T
    modes = []
    for c in range(3):
        m = np.zeros((X.shape[0], 3)); m[:, c] = 1.0; modes.append(m.ravel())
    for (a, b) in ((0, 1), (1, 2), (0, 2)):
        m = np.zeros((X.shape[0], 3)); m[:, a] = -X[:, b]; m[:, b] = X[:, a]
        modes.append(m.ravel())
    scale = np.abs(K).max()
    for m in modes:
        assert np.abs(K @ m).max() < 1e-10 * scale
    assert np.linalg.eigvalsh(K).min() > -1e-9 * scale


# ------------------------------------------------------------------ GPU parity
# Gauss-Legendre rules of GaussLegendre.f90:41-153 (orders 1..9, the
# standard published nodes and weights to 30 significant digits): upper-half
# nodes (ascending, x >= 0) and weights; order 3's weights are the divisions
# 8/9 and 5/9.
GL_TABLE = {
    1: (["0.0"], ["2.0"]),
    2: (["0.577350269189625764509148780502"], ["1.0"]),
    3: (["0.0", "0.774596669241483377035853079956"], [8.0 / 9.0, 5.0 / 9.0]),
    4: (["0.339981043584856264802665759103", "0.861136311594052575223946488893"],
        ["0.652145154862546142626936050778", "0.347854845137453857373063949222"]),
    5: (["0.0", "0.538469310105683091036314420700", "0.906179845938663992797626878299"],
        ["0.568888888888888888888888888889", "0.478628670499366468041291514836",
         "0.236926885056189087514264040720"]),
    6: (["0.238619186083196908630501721681", "0.661209386466264513661399595020",
         "0.932469514203152027812301554494"],
        ["0.467913934572691047389870343990", "0.360761573048138607569833513838",
         "0.171324492379170345040296142173"]),
    7: (["0.0", "0.405845151377397166906606412077", "0.741531185599394439863864773281",
         "0.949107912342758524526189684048"],
        ["0.417959183673469387755102040816", "0.381830050505118944950369775489",
         "0.279705391489276667901467771424", "0.129484966168869693270611432679"]),
    8: (["0.183434642495649804939476142360", "0.525532409916328985817739049189",
         "0.796666477413626739591553936476", "0.960289856497536231683560868569"],
        ["0.362683783378361982965150449277", "0.313706645877887287337962201987",
         "0.222381034453374470544355994426", "0.101228536290376259152531354310"]),
    9: (["0.0", "0.324253423403808929038538014643", "0.613371432700590397308702039341",
         "0.836031107326635794299429788070", "0.968160239507626089835576202904"],
        ["0.330239355001259763164525069287", "0.312347077040002840068630406584",
         "0.260610696402935462318742869419", "0.180648160694857404058472031243",
         "0.812743883615744119718921581105E-01"]),
}


@pytest.mark.parametrize("n", range(1, 10))
def test_oracle_gauss_rule_is_the_reference_table_bit_for_bit(n):
    """The oracle's rule (the one the GPU assembly's parity tests compare
    with bit for bit) equals the reference's table, each literal rounded to
    double as a Fortran compiler rounds it (Python's float is correctly
    rounded)."""
    import ctypes
    xs, ws = GL_TABLE[n]
    up_x = [float(v) for v in xs]
    up_w = [float(v) for v in ws]
    if n % 2:
        ref_x = [-v for v in up_x[:0:-1]] + up_x
        ref_w = up_w[:0:-1] + up_w
    else:
        ref_x = [-v for v in up_x[::-1]] + up_x
        ref_w = up_w[::-1] + up_w
    x = np.zeros(n)
    w = np.zeros(n)
    f = oracle.lib().oracle_gauss_legendre
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    f(n, x.ctypes.data, w.ctypes.data)
    assert x.tobytes() == np.array(ref_x).tobytes()
    assert w.tobytes() == np.array(ref_w).tobytes()


def _gpu_vs_oracle(name):
    from yeti_b200.stiffmtrx_elemstorage import sys_linmat_lindef_static
    d, args = load_fixture(name)
    ref = oracle.sys_linmat_lindef_static(*args)
    got = sys_linmat_lindef_static(*args)
    return d, ref, got


@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES)
def test_gpu_coo_matches_oracle(cuda_ok, name):
    d, (k0, r0, c0, f0), (k1, r1, c1, f1) = _gpu_vs_oracle(name)
    assert k1.dtype == np.float64 and r1.dtype == np.int32 and c1.dtype == np.int32
    assert k1.shape == k0.shape
    np.testing.assert_array_equal(r1, r0)
    np.testing.assert_array_equal(c1, c0)
    assert np.linalg.norm(k1 - k0) <= TOL * np.linalg.norm(k0)
    assert np.abs(k1 - k0).max() <= TOL * np.abs(k0).max()
    # the FP64 kernels follow the reference's operation order without FMA
    # contraction: the COO values and the load vector are bit-identical
    np.testing.assert_array_equal(k1, k0)
    np.testing.assert_array_equal(f1, f0)
    if np.linalg.norm(f0) > 0:
        assert np.linalg.norm(f1 - f0) <= TOL * np.linalg.norm(f0)
    else:
        assert np.linalg.norm(f1) == 0.0
    if int(d["nb_dof_free"]) < int(d["nb_dof_tot"]) and np.linalg.norm(f0) > 0:
        s0 = _solve(d, k0, r0, c0, f0)
        s1 = _solve(d, k1, r1, c1, f1)
        assert np.linalg.norm(s1 - s0) <= TOL * np.linalg.norm(s0)


@pytest.mark.gpu
def test_gpu_coo_device_output_and_inactive_elements(cuda_ok):
    """Device-resident outputs, and slots compacted over active elements."""
    import torch
    from yeti_b200.stiffmtrx_elemstorage import sys_linmat_lindef_static
    d, args = load_fixture("cantilever_p2_16x4x4")
    active = np.ones(int(d["nb_elem"]), dtype=np.int64)
    active[::3] = 0
    nb_data = int(active.sum()) * 3321
    args = list(args)
    args[0] = active
    args[1] = nb_data
    k0, r0, c0, f0 = oracle.sys_linmat_lindef_static(*args)
    k1, r1, c1, f1 = sys_linmat_lindef_static(*args, device_out=True)
    assert k1.is_cuda and k1.numel() == nb_data
    np.testing.assert_array_equal(r1.cpu().numpy(), r0)
    np.testing.assert_array_equal(c1.cpu().numpy(), c0)
    k1 = k1.cpu().numpy()
    assert np.linalg.norm(k1 - k0) <= TOL * np.linalg.norm(k0)
    f1 = f1.cpu().numpy()
    assert np.linalg.norm(f1 - f0) <= TOL * np.linalg.norm(f0)
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_gpu_rejects_unsupported_element(cuda_ok):
    from yeti_b200._lib import YetiError
    from yeti_b200.stiffmtrx_elemstorage import sys_linmat_lindef_static
    d, args = load_fixture("grad_unit_cube")
    args = list(args)
    args[10] = "U3"   # shell patch
    with pytest.raises(YetiError):
        sys_linmat_lindef_static(*args)


# ------------------------------------------- sum-factorised element kernel
# Synthetic U1 cubes beyond the fixtures' degree 2: (elements, degrees,
# perturbation, weight range).  Mixed degrees keep one Gauss count per
# direction (max p + 1), as the reference's NBINT does.
SF_PATCHES = {
    "p3_3x3x2": ((3, 3, 2), 3, 0.2, (0.8, 1.2)),
    "p4_2x2x2": ((2, 2, 2), 4, 0.1, (0.8, 1.2)),
    "p234_2x3x2": ((2, 3, 2), (2, 3, 4), 0.15, (0.9, 1.1)),
    "p5_2x1x1": ((2, 1, 1), 5, 0.1, None),
}


def _sf_args(name):
    from yeti_b200.patches import cube_patch, u1_system_args
    nel, p, pert, wr = SF_PATCHES[name]
    return u1_system_args(cube_patch(nel, p, perturb=pert, wrange=wr, seed=11), E=210.0, nu=0.3)


def test_u1_system_args_match_the_reference_layout():
    """The synthetic model builder reproduces the IEN / Nijk / weight / knot
    layout that the reference's preprocessing wrote for the p=2 cantilever."""
    from yeti_b200.patches import u1_system_args
    from yeti_b200.stiffmtrx_elemstorage import SYSTEM_ARG_NAMES
    d, args = load_fixture("cantilever_p2_16x4x4")
    mine = u1_system_args({"p": (2, 2, 2), "nel": (16, 4, 4), "cps": np.asarray(d["COORDS3D"]),
                           "weights": np.ones(int(d["nb_cp"]))}, E=210000.0, nu=0.3)
    for name, a, b in zip(SYSTEM_ARG_NAMES, args, mine):
        if name in ("activeElement", "IEN", "Nkv", "Ukv", "Nijk", "weight", "Jpqr", "NBINT", "NNODE",
                    "MATERIAL_PROPERTIES", "nb_elem", "nb_cp", "nb_dof_tot"):
            np.testing.assert_array_equal(np.asarray(a).ravel(), np.asarray(b).ravel(), err_msg=name)
    k0 = oracle.sys_linmat_lindef_static(*args)[0]
    k1 = oracle.sys_linmat_lindef_static(*mine)[0]
    np.testing.assert_array_equal(k0, k1)


def _check_close(k0, r0, c0, k1, r1, c1):
    np.testing.assert_array_equal(r1, r0)
    np.testing.assert_array_equal(c1, c0)
    assert np.linalg.norm(k1 - k0) <= TOL * np.linalg.norm(k0)
    assert np.abs(k1 - k0).max() <= TOL * np.abs(k0).max()


@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES)
def test_gpu_sumfact_matches_oracle_on_fixtures(cuda_ok, name):
    from yeti_b200.stiffmtrx_elemstorage import sys_linmat_lindef_static
    d, args = load_fixture(name)
    k0, r0, c0, f0 = oracle.sys_linmat_lindef_static(*args)
    k1, r1, c1, f1 = sys_linmat_lindef_static(*args, element_kernel="sumfact")
    _check_close(k0, r0, c0, k1, r1, c1)
    np.testing.assert_array_equal(f1, f0)   # the load vector is the same kernel's
    if int(d["nb_dof_free"]) < int(d["nb_dof_tot"]) and np.linalg.norm(f0) > 0:
        s0 = _solve(d, k0, r0, c0, f0)
        s1 = _solve(d, k1, r1, c1, f1)
        # values equal to rounding (not bit for bit): the displacement moves
        # by up to cond(K) times that; 1e-10 on these models (measured
        # 1.5e-12 on the slender p=2 cantilever)
        assert np.linalg.norm(s1 - s0) <= 1e-10 * np.linalg.norm(s0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SF_PATCHES))
def test_gpu_sumfact_and_pairs_match_oracle_beyond_degree_two(cuda_ok, name):
    from yeti_b200.stiffmtrx_elemstorage import sys_linmat_lindef_static
    args = _sf_args(name)
    k0, r0, c0, _ = oracle.sys_linmat_lindef_static(*args)
    k1, r1, c1, _ = sys_linmat_lindef_static(*args, element_kernel="sumfact")
    _check_close(k0, r0, c0, k1, r1, c1)
    k2, r2, c2, _ = sys_linmat_lindef_static(*args)
    np.testing.assert_array_equal(k2, k0)
    np.testing.assert_array_equal(r2, r0)
    np.testing.assert_array_equal(c2, c0)


@pytest.mark.gpu
def test_gpu_sumfact_rejects_a_partial_gauss_rule(cuda_ok):
    from yeti_b200._lib import YetiError
    from yeti_b200.patches import cube_patch, u1_system_args
    from yeti_b200.stiffmtrx_elemstorage import sys_linmat_lindef_static
    args = u1_system_args(cube_patch((2, 2, 2), 2), nbint=26)
    with pytest.raises(YetiError, match="EUNSUPPORTED"):
        sys_linmat_lindef_static(*args, element_kernel="sumfact")
    with pytest.raises(ValueError):
        sys_linmat_lindef_static(*args, element_kernel="fast")


@pytest.mark.gpu
def test_gpu_context_times_the_element_kernels(cuda_ok):
    from yeti_b200._lib import Context
    from yeti_b200.stiffmtrx_elemstorage import sys_linmat_lindef_static
    args = _sf_args("p3_3x3x2")
    ctx = Context(0)
    assert ctx.kernel_ms("k_u1_stiffness") is None
    ctx.set_timing(True)
    sys_linmat_lindef_static(*args, ctx=ctx)
    sys_linmat_lindef_static(*args, ctx=ctx, element_kernel="sumfact")
    t_pairs, t_sf = ctx.kernel_ms("k_u1_stiffness"), ctx.kernel_ms("k_u1_stiffness_sf")
    assert t_pairs is not None and t_pairs > 0 and t_sf is not None and t_sf > 0
    ctx.set_timing(False)
    assert ctx.kernel_ms("k_u1_stiffness") is None
    sys_linmat_lindef_static(*args, ctx=ctx)
    assert ctx.kernel_ms("k_u1_stiffness") is None
    ctx.close()


def test_u1_system_args_reproduce_the_cantilever_loads_and_clamps():
    """With the clamp and face-load options the builder writes the loads,
    boundary conditions and free-dof list the reference's preprocessing
    wrote for the p=2 cantilever (U23 on the face x=10, clamped x=0)."""
    from yeti_b200.patches import u1_system_args
    from yeti_b200.stiffmtrx_elemstorage import SYSTEM_ARG_NAMES
    d, args = load_fixture("cantilever_p2_16x4x4")
    mine = u1_system_args({"p": (2, 2, 2), "nel": (16, 4, 4), "cps": np.asarray(d["COORDS3D"]),
                           "weights": np.ones(int(d["nb_cp"]))}, E=210000.0, nu=0.3,
                          clamp_u0=True, load_u1=(3, -1.0))
    for name, a, b in zip(SYSTEM_ARG_NAMES, args, mine):
        if name in ("indDLoad", "JDLType", "ADLMAG", "load_target_nbelem", "bc_values",
                    "bc_target", "bc_target_nbelem", "ind_dof_free", "nb_dof_free", "nb_bc",
                    "nb_load"):
            np.testing.assert_array_equal(np.asarray(a).ravel(), np.asarray(b).ravel(), err_msg=name)
    k0, _, _, f0 = oracle.sys_linmat_lindef_static(*args)
    k1, _, _, f1 = oracle.sys_linmat_lindef_static(*mine)
    np.testing.assert_array_equal(k0, k1)
    np.testing.assert_array_equal(f0, f1)
