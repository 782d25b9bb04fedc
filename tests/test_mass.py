"""Consistent mass matrix of U1 solids (build_CMASSMatrix,
src/yeti_iga/main/compute_CMASSMatrix.f, with UMASSMAT_byCP's U1 branch).

Bars: the oracle's total mass t^T M t of a rigid translation t equals
rho x the oracle volume within 1e-13 (partition of unity), its COO rows and
columns are the stiffness assembly's, and the GPU matrix equals the oracle's
bit for bit (host and device outputs).
"""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from conftest import load_fixture
from yeti_b200.stiffmtrx_elemstorage import SYSTEM_ARG_NAMES

FIXTURES = ["grad_unit_cube", "cantilever_p2_16x4x4", "quarter_annulus_p2_4x4x2",
            "quarter_annulus_p2_32x32x2"]


def mass_inputs(name, rho=7.85):
    """The get_inputs4massmat list (IGA_parametrization.py:1756-1762) of a
    fixture model with density rho on every patch; also returns the
    fixture's system arguments."""
    _, args = load_fixture(name)
    d = dict(zip(SYSTEM_ARG_NAMES, args))
    npatch = np.atleast_1d(d["nb_elem_patch"]).size
    inputs = [d["activeElement"], d["nb_data"], np.asarray(d["COORDS3D"], dtype=np.float64),
              d["IEN"], d["nb_elem_patch"], d["Nkv"], d["Ukv"], d["Nijk"], d["weight"],
              d["Jpqr"], d["ELT_TYPE"], d["PROPS"], d["JPROPS"], np.full(npatch, rho),
              d["TENSOR"], d["ind_dof_free"], d["nb_dof_free"], d["MCRD"], d["NBINT"],
              d["NNODE"]]
    return inputs, args, d


def _full(data, row, col, n):
    side = sp.coo_matrix((data, (row, col)), shape=(n, n)).tocsr()
    return side + side.T


# ---------------------------------------------------------------------- CPU
@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_total_mass_and_slots(name):
    rho = 7.85
    inputs, args, d = mass_inputs(name, rho)
    md, mr, mc = oracle.build_cmassmatrix(inputs)
    X = inputs[2]
    n = 3 * X.shape[1]
    M = _full(md, mr, mc, n)
    area = [np.ones(np.atleast_1d(d["nb_elem_patch"]).size, dtype=np.int64), X, d["IEN"],
            d["nb_elem_patch"], d["Nkv"], d["Ukv"], d["Nijk"], d["weight"], d["Jpqr"],
            d["ELT_TYPE"], d["PROPS"], d["JPROPS"], d["TENSOR"], d["MCRD"], d["NBINT"],
            d["NNODE"]]
    if np.all(np.asarray(d["activeElement"]) == 1):
        v, _ = oracle.volume(area, gradient=False)
        for c in range(3):
            t = np.zeros(n)
            t[c::3] = 1.0
            assert abs(t @ (M @ t) - rho * v) <= 1e-13 * rho * v
    _, kr, kc, _ = oracle.sys_linmat_lindef_static(*args)
    assert np.array_equal(mr, kr) and np.array_equal(mc, kc)


# ---------------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES)
def test_mass_matrix_matches_oracle(cuda_ok, name):
    from yeti_b200.massmtrx import build_cmassmatrix
    inputs, _, _ = mass_inputs(name)
    md0, mr0, mc0 = oracle.build_cmassmatrix(inputs)
    md, mr, mc = build_cmassmatrix(*inputs)
    assert np.array_equal(mr, mr0) and np.array_equal(mc, mc0)
    assert np.array_equal(md, md0)
    dd, dr, dc = build_cmassmatrix(*inputs, device_out=True)
    assert np.array_equal(dd.cpu().numpy(), md0)
    assert np.array_equal(dr.cpu().numpy(), mr0) and np.array_equal(dc.cpu().numpy(), mc0)


@pytest.mark.gpu
@pytest.mark.parametrize("deg", [4, 5])
def test_mass_matrix_matches_oracle_with_gauss_chunks(cuda_ok, deg):
    """Degrees whose Gauss points do not fit shared memory at once (125 and
    216 points per element): the kernel resumes each pair's running sum
    across point chunks, so the entries stay bit-identical."""
    from yeti_b200.massmtrx import build_cmassmatrix
    from yeti_b200.patches import cube_patch, u1_system_args
    args = u1_system_args(cube_patch((2, 1, 1), deg, perturb=0.1, wrange=(0.8, 1.2), seed=5))
    d = dict(zip(SYSTEM_ARG_NAMES, args))
    inputs = [d["activeElement"], d["nb_data"], np.asarray(d["COORDS3D"], dtype=np.float64),
              d["IEN"], d["nb_elem_patch"], d["Nkv"], d["Ukv"], d["Nijk"], d["weight"],
              d["Jpqr"], d["ELT_TYPE"], d["PROPS"], d["JPROPS"], np.full(1, 2.5),
              d["TENSOR"], d["ind_dof_free"], d["nb_dof_free"], d["MCRD"], d["NBINT"],
              d["NNODE"]]
    md0, mr0, mc0 = oracle.build_cmassmatrix(inputs)
    md, mr, mc = build_cmassmatrix(*inputs)
    assert np.array_equal(mr, mr0) and np.array_equal(mc, mc0)
    assert np.array_equal(md, md0)
