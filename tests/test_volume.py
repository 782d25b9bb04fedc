"""Volume of U1 patches and its shape gradient (computeVolume /
computeGradVolume, src/yeti_iga/optim/volume.f90, gradvolume.f90).

Bars: the oracle reproduces the known volumes (unit cube, 10x1x1 beam,
quarter annulus pi (4^2 - 1^2) / 4 x 0.1 up to its quadrature error); its
gradient matches central finite differences (step 1e-6, FP64) on 20 seeded
coordinates within 1e-6 relative, sums to zero over the control points
(translation) and satisfies sum_k P_k . dV/dP_k = 3 V (cubic scaling); the
GPU volume and gradient equal the oracle's bit for bit.
"""
import numpy as np
import pytest

import oracle
from conftest import load_fixture
from yeti_b200.stiffmtrx_elemstorage import SYSTEM_ARG_NAMES

FIXTURES = ["grad_unit_cube", "cantilever_p2_16x4x4", "quarter_annulus_p2_4x4x2",
            "quarter_annulus_p2_32x32x2"]
EXACT = {"grad_unit_cube": (1.0, 1e-14), "cantilever_p2_16x4x4": (10.0, 1e-13),
         "quarter_annulus_p2_4x4x2": (np.pi * 15.0 / 4.0 * 0.1, 1e-8),
         "quarter_annulus_p2_32x32x2": (np.pi * 15.0 / 4.0 * 0.1, 1e-12)}


def area_inputs(name):
    """The get_inputs4area list (IGA_parametrization.py:1306-1310) of a
    fixture model, every patch listed."""
    _, args = load_fixture(name)
    d = dict(zip(SYSTEM_ARG_NAMES, args))
    npatch = np.atleast_1d(d["nb_elem_patch"]).size
    return [np.ones(npatch, dtype=np.int64), np.asarray(d["COORDS3D"], dtype=np.float64),
            d["IEN"], d["nb_elem_patch"], d["Nkv"], d["Ukv"], d["Nijk"], d["weight"],
            d["Jpqr"], d["ELT_TYPE"], d["PROPS"], d["JPROPS"], d["TENSOR"], d["MCRD"],
            d["NBINT"], d["NNODE"]]


# ---------------------------------------------------------------------- CPU
@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_volume_known_values(name):
    v, _ = oracle.volume(area_inputs(name), gradient=False)
    exact, tol = EXACT[name]
    assert abs(v - exact) <= tol * exact


@pytest.mark.parametrize("name", ["grad_unit_cube", "quarter_annulus_p2_4x4x2"])
def test_oracle_gradient_finite_differences_and_invariants(name):
    A = area_inputs(name)
    X = A[1]
    v, g = oracle.volume(A)
    gmax = np.abs(g).max()
    # translation: the volume does not move, the gradient sums to zero
    assert np.abs(g.sum(axis=1)).max() <= 1e-12 * gmax * X.shape[1]
    # cubic scaling: sum_k P_k . dV/dP_k = 3 V
    assert abs((X * g).sum() - 3.0 * v) <= 1e-12 * v
    rng = np.random.default_rng(20)
    h = 1e-6
    for _ in range(20):
        c, k = int(rng.integers(3)), int(rng.integers(X.shape[1]))
        Ap, Am = list(A), list(A)
        Ap[1] = X.copy()
        Ap[1][c, k] += h
        Am[1] = X.copy()
        Am[1][c, k] -= h
        fd = (oracle.volume(Ap, False)[0] - oracle.volume(Am, False)[0]) / (2 * h)
        assert abs(fd - g[c, k]) <= 1e-6 * gmax


# ---------------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES)
def test_volume_and_gradient_match_oracle(cuda_ok, name):
    from yeti_b200.volume import computegradvolume, computevolume
    A = area_inputs(name)
    v0, g0 = oracle.volume(A)
    assert computevolume(*A) == v0
    g = computegradvolume(*A)
    assert g.shape == g0.shape
    assert np.array_equal(g, g0)


@pytest.mark.gpu
def test_unlisted_patch_contributes_nothing(cuda_ok):
    from yeti_b200.volume import volume_and_gradient
    A = area_inputs("grad_unit_cube")
    A[0] = np.zeros_like(A[0])
    v, g = volume_and_gradient(A)
    assert v == 0.0 and not g.any()


@pytest.mark.gpu
def test_volume_autograd_function(cuda_ok):
    import torch
    from yeti_b200.volume import Volume, computegradvolume
    A = area_inputs("quarter_annulus_p2_4x4x2")
    P = torch.tensor(A[1], dtype=torch.float64, requires_grad=True)
    V = Volume.apply(P, A)
    V.backward()
    assert np.array_equal(P.grad.numpy(), computegradvolume(*A))
    assert abs(V.item() - oracle.volume(A, False)[0]) == 0.0
