"""yeti_wq_apply_static: K u with host buffers and no device allocation.

Callers that cannot allocate device memory at the point of the call (all
device memory reserved up front by another allocator, or a latency-critical
loop that must not pay cudaMalloc/cudaFree's implicit synchronisation) use
this entry point; it stages the vectors in a fixed device array (at most
2,097,152 dofs per vector) shared by all calls.  Checked through the C ABI
against yeti_wq_apply (host buffers) on two calls in a row, within the
tolerance of the other WQ tests (1e-12 relative, FP64; 2e-6, FP32), for a
degree-3 operator (streaming apply) and a degree-6 one (element-block apply),
with FP64 and FP32 calls alternating so that the shared bytes are reused at
both widths.

This file is named to be collected last.
"""
import numpy as np
import pytest

from yeti_b200.patches import cube_patch


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.gpu
@pytest.mark.parametrize("p,nel", [(3, (6, 5, 7)), (6, (2, 3, 2))])
def test_static_apply_matches_allocating_apply_twice(cuda_ok, p, nel):
    from yeti_b200._lib import MEM_HOST, PREC_F32, PREC_F64, check, lib, ptr
    from yeti_b200.wq import WQElasticity
    P = cube_patch(nel, (p, p, p), perturb=0.2, wrange=(0.8, 1.2), seed=9)
    op = WQElasticity(P, 1.0, 0.3, {"w0": (0, 1, 2)})
    L = lib()
    rng = np.random.default_rng(3)
    for call in range(2):   # the shared array keeps the last call's contents
        u = rng.standard_normal(op.ndof)
        ref = np.empty_like(u)
        check(L.yeti_wq_apply(op.handle, ptr(u), ptr(ref), PREC_F64, MEM_HOST),
              "yeti_wq_apply")
        got = np.empty_like(u)
        check(L.yeti_wq_apply_static(op.handle, ptr(u), ptr(got), PREC_F64),
              "yeti_wq_apply_static")
        assert _rel(got, ref) < 1e-12, call
        u32 = u.astype(np.float32)
        ref32 = np.empty_like(u32)
        check(L.yeti_wq_apply(op.handle, ptr(u32), ptr(ref32), PREC_F32, MEM_HOST),
              "yeti_wq_apply")
        got32 = np.empty_like(u32)
        check(L.yeti_wq_apply_static(op.handle, ptr(u32), ptr(got32), PREC_F32),
              "yeti_wq_apply_static")
        assert _rel(got32.astype(np.float64), ref32.astype(np.float64)) < 2e-6, call


@pytest.mark.gpu
def test_static_apply_reports_a_wait_that_gave_up(cuda_ok):
    """A bounded wait of the streaming apply that runs out (the wait limit is
    set to 0 polls: the first wait of every CTA gives up at once, after which
    the kernel lets its copy in flight land and returns) is reported as
    YETI_ETIMEDOUT by the static entry as by yeti_wq_apply; with the default
    limit restored, the next calls succeed and agree."""
    from yeti_b200._lib import MEM_HOST, PREC_F32, check, lib, ptr
    from yeti_b200.wq import WQElasticity
    P = cube_patch((6, 5, 7), (3, 3, 3), perturb=0.2, wrange=(0.8, 1.2), seed=9)
    op = WQElasticity(P, 1.0, 0.3, {"w0": (0, 1, 2)})
    L = lib()
    u = np.random.default_rng(4).standard_normal(op.ndof).astype(np.float32)
    out = np.empty_like(u)
    check(L.yeti_wq_set_wait_limit(op.handle, 0), "yeti_wq_set_wait_limit")
    assert L.yeti_wq_apply(op.handle, ptr(u), ptr(out), PREC_F32, MEM_HOST) == -5
    assert L.yeti_wq_apply_static(op.handle, ptr(u), ptr(out), PREC_F32) == -5
    assert b"gave up" in L.yeti_last_error()
    check(L.yeti_wq_set_wait_limit(op.handle, -1), "yeti_wq_set_wait_limit")
    ref = np.empty_like(u)
    check(L.yeti_wq_apply(op.handle, ptr(u), ptr(ref), PREC_F32, MEM_HOST), "yeti_wq_apply")
    got = np.empty_like(u)
    check(L.yeti_wq_apply_static(op.handle, ptr(u), ptr(got), PREC_F32),
          "yeti_wq_apply_static")
    assert _rel(got.astype(np.float64), ref.astype(np.float64)) < 2e-6


@pytest.mark.gpu
def test_static_apply_rejects_operators_beyond_the_limit(cuda_ok):
    from yeti_b200._lib import PREC_F64, lib, ptr
    from yeti_b200.wq import WQElasticity
    # 102 x 102 x 70 control points x 3 = 2,184,840 dofs > 2,097,152
    P = cube_patch((100, 100, 68), (2, 2, 2))
    op = WQElasticity(P, 1.0, 0.3, precisions="f64")
    assert op.ndof > 2097152
    u = np.zeros(op.ndof)
    out = np.zeros(op.ndof)
    rc = lib().yeti_wq_apply_static(op.handle, ptr(u), ptr(out), PREC_F64)
    assert rc == -1
    assert b"static staging limit" in lib().yeti_last_error()
