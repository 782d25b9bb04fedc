"""Models of several U1 patches (different degrees, element counts and
materials per patch): the per-patch loops of the assembly, mass matrix,
shape gradient and volume (build_system_elemStorage.f90:24-315 and the
optim routines iterate over patches the same way).

Bars: the oracle's two-patch COO equals the two one-patch assemblies placed
one after the other (slots compacted per patch, rows and columns of the
second patch shifted by its control-point offset); on the GPU the pair
kernel, the mass matrix, the gradient and the volume equal the oracle bit
for bit, the sum-factorised kernel within 1e-12.
"""
import numpy as np
import pytest

import oracle
from yeti_b200.patches import cube_patch, u1_system_args, u1_system_args_multi
from yeti_b200.stiffmtrx_elemstorage import SYSTEM_ARG_NAMES

MATERIALS = [(210.0, 0.3), (70.0, 0.25), (1.0, 0.35)]


def _patches():
    return [cube_patch((3, 2, 2), 2, perturb=0.1, wrange=(0.9, 1.1), seed=1),
            cube_patch((2, 2, 3), (3, 2, 3), size=(1.0, 2.0, 1.5), perturb=0.1,
                       wrange=(0.9, 1.1), seed=2),
            cube_patch((2, 2, 2), 4, size=(0.5, 0.5, 0.5), perturb=0.05, seed=3)]


def _dict(args):
    return dict(zip(SYSTEM_ARG_NAMES, args))


def _mass_inputs(args, rho=7.85):
    d = _dict(args)
    npatch = np.atleast_1d(d["nb_elem_patch"]).size
    return [d["activeElement"], d["nb_data"], np.asarray(d["COORDS3D"], dtype=np.float64),
            d["IEN"], d["nb_elem_patch"], d["Nkv"], d["Ukv"], d["Nijk"], d["weight"],
            d["Jpqr"], d["ELT_TYPE"], d["PROPS"], d["JPROPS"], np.full(npatch, rho),
            d["TENSOR"], d["ind_dof_free"], d["nb_dof_free"], d["MCRD"], d["NBINT"],
            d["NNODE"]]


def _area_inputs(args):
    d = _dict(args)
    npatch = np.atleast_1d(d["nb_elem_patch"]).size
    return [np.ones(npatch, dtype=np.int64), np.asarray(d["COORDS3D"], dtype=np.float64),
            d["IEN"], d["nb_elem_patch"], d["Nkv"], d["Ukv"], d["Nijk"], d["weight"],
            d["Jpqr"], d["ELT_TYPE"], d["PROPS"], d["JPROPS"], d["TENSOR"], d["MCRD"],
            d["NBINT"], d["NNODE"]]


# ---------------------------------------------------------------------- CPU
def test_oracle_multipatch_is_the_patches_one_after_the_other():
    patches = _patches()
    args = u1_system_args_multi(patches, MATERIALS)
    k, r, c, _ = oracle.sys_linmat_lindef_static(*args)
    o_slot, o_cp = 0, 0
    for P, (E, nu) in zip(patches, MATERIALS):
        a1 = u1_system_args(P, E=E, nu=nu)
        k1, r1, c1, _ = oracle.sys_linmat_lindef_static(*a1)
        n = k1.size
        np.testing.assert_array_equal(k[o_slot:o_slot + n], k1)
        np.testing.assert_array_equal(r[o_slot:o_slot + n], r1 + 3 * o_cp)
        np.testing.assert_array_equal(c[o_slot:o_slot + n], c1 + 3 * o_cp)
        o_slot += n
        o_cp += int(a1[36])
    assert o_slot == k.size


# ---------------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_gpu_multipatch_assembly_both_kernels(cuda_ok):
    from yeti_b200.stiffmtrx_elemstorage import sys_linmat_lindef_static
    args = u1_system_args_multi(_patches(), MATERIALS)
    k0, r0, c0, f0 = oracle.sys_linmat_lindef_static(*args)
    k1, r1, c1, f1 = sys_linmat_lindef_static(*args)
    np.testing.assert_array_equal(k1, k0)
    np.testing.assert_array_equal(r1, r0)
    np.testing.assert_array_equal(c1, c0)
    np.testing.assert_array_equal(f1, f0)
    k2, r2, c2, _ = sys_linmat_lindef_static(*args, element_kernel="sumfact")
    np.testing.assert_array_equal(r2, r0)
    np.testing.assert_array_equal(c2, c0)
    assert np.abs(k2 - k0).max() <= 1e-12 * np.abs(k0).max()


@pytest.mark.gpu
def test_gpu_multipatch_mass_matrix(cuda_ok):
    from yeti_b200.massmtrx import build_cmassmatrix
    inputs = _mass_inputs(u1_system_args_multi(_patches(), MATERIALS))
    m0, r0, c0 = oracle.build_cmassmatrix(inputs)
    m1, r1, c1 = build_cmassmatrix(*inputs)
    np.testing.assert_array_equal(m1, m0)
    np.testing.assert_array_equal(r1, r0)
    np.testing.assert_array_equal(c1, c0)


@pytest.mark.gpu
def test_gpu_multipatch_gradient_and_volume(cuda_ok):
    from yeti_b200.gradient import grad_from_system_args
    from yeti_b200.volume import volume_and_gradient
    args = u1_system_args_multi(_patches(), MATERIALS)
    nb_cp = int(args[36])
    rng = np.random.default_rng(5)
    sol = rng.standard_normal((3, nb_cp))
    adj = rng.standard_normal((2, 3, nb_cp))
    gi, ge = grad_from_system_args(args, sol, adj)
    oi, oe = oracle.grad_lin_elast_work(args, sol, adj)
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(ge, oe)
    A = _area_inputs(args)
    v1, g1 = volume_and_gradient(A)
    v0, g0 = oracle.volume(A)
    assert v1 == v0
    np.testing.assert_array_equal(g1, g0)
