"""GPU parity of the WQ operator at the benchmark sizes, against the oracle.

The two benchmark patches, built exactly as bench.py builds them:
* 64^3 elements, p=3, unit cube, interior control points perturbed
  U(-0.2h, 0.2h), weights U(0.8, 1.2), seed 20261203, clamped at w=0
  (902,289 dofs, 2,352,637 WQ points);
* 128 x 128 x 32 elements, p=4, block 4 x 4 x 1, perturbed U(-0.1h, 0.1h),
  weights U(0.8, 1.2), seed 20261208, clamped at w=0 (1,881,792 dofs,
  4,910,999 WQ points).

At these sizes the streaming apply runs its regular-tile walks, the boundary
tiles of both ends and the CTA segment splits that small cases never reach.
Bars as in test_wq.py: FP64 apply, diagonal and body force within 1e-12
(relative 2-norm) of the FP64 oracle, FP32 apply within 2e-6.  The mixed
solve of the 64^3 block (rtol 1e-9, the bench's) is checked on the oracle's
side: its residual under the oracle's operator is below 1e-8 of the load.
The oracle needs about 6 GB (64^3) and 13 GB (p=4 block) of host memory.
"""
import numpy as np
import pytest

from yeti_b200.patches import cube_patch

SEED = 20261203
CONFIGS = {
    "p3_64cube": dict(nel=(64, 64, 64), p=3, size=(1.0, 1.0, 1.0), perturb=0.2, seed=SEED),
    "p4_128x128x32": dict(nel=(128, 128, 32), p=4, size=(4.0, 4.0, 1.0), perturb=0.1,
                          seed=SEED + 5),
}
CLAMP = {"w0": (0, 1, 2)}


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module", params=list(CONFIGS))
def pair(request, cuda_ok):
    from oracle.wq_ops import WQOracle
    from yeti_b200.wq import WQElasticity
    c = CONFIGS[request.param]
    P = cube_patch(c["nel"], c["p"], size=c["size"], perturb=c["perturb"], wrange=(0.8, 1.2),
                   seed=c["seed"])
    op = WQElasticity(P, 1.0, 0.3, CLAMP, precisions="both")
    ref = WQOracle(P, 1.0, 0.3, CLAMP)
    yield request.param, op, ref
    del op


@pytest.mark.gpu
def test_fullsize_apply_fp64_fp32(pair):
    name, op, ref = pair
    rng = np.random.default_rng(7)
    for _ in range(2):
        u = rng.standard_normal(op.ndof) * op.free_mask
        k0 = ref.apply(u)
        assert _rel(op.eval_Ku(u), k0) < 1e-12, name
        k32 = op.eval_Ku(u.astype(np.float32), precision="f32").astype(np.float64)
        assert _rel(k32, k0) < 2e-6, name


@pytest.mark.gpu
def test_fullsize_diagonal_and_body_force(pair):
    name, op, ref = pair
    assert _rel(op.diag(), ref.diag()) < 1e-12, name
    f = [0.0, 0.0, -1.0]
    assert _rel(op.eval_bodyforce_vector(f), ref.body_force(f)) < 1e-12, name


@pytest.mark.gpu
def test_fullsize_mixed_solve_residual_under_oracle(pair):
    name, op, ref = pair
    if name != "p3_64cube":
        pytest.skip("one solve suffices: the p=4 block's apply is pinned above")
    import torch
    b = op.eval_bodyforce_vector([0.0, 0.0, -1.0])
    x, st = op.pcg(torch.from_numpy(b).cuda(), rtol=1e-9, mixed=True)
    x = x.cpu().numpy()
    m = op.free_mask
    r = (b - ref.apply(x)) * m
    assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(b * m), st
