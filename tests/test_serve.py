"""Serving loop (yeti_serve_*): results do not depend on what else is being
served, admission honours the HBM budget, and the loop overlaps requests.

Tolerances: each solve stops at ||r|| <= 1e-10 ||b||; a request's solution
served alone and served in a mix of other patches must agree to 1e-8
relative (the only difference is the order of floating-point atomics in the
operator apply), and must match the one-shot FP64 solver (WQElasticity.pcg)
to 1e-8 relative.
"""
import numpy as np
import pytest

from yeti_b200.patches import cube_patch


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _request(nel, p, seed, nrhs):
    patch = cube_patch(nel, p, perturb=0.15, wrange=(0.9, 1.1), seed=seed)
    ndof = 3 * int(np.prod([p + n for n in nel]))
    rhs = np.random.default_rng(seed + 1).standard_normal((nrhs, ndof))
    return patch, rhs


def test_synthetic_requests_are_seeded():
    from yeti_b200.serve import synthetic_requests
    a = synthetic_requests(5, seed=3)
    b = synthetic_requests(5, seed=3)
    assert [r["ndof"] for r in a] == [r["ndof"] for r in b]
    assert all(r["patch"]["p"][0] in (2, 3) for r in a)
    assert all(4 <= n <= 32 for r in a for n in r["patch"]["nel"])
    assert all(1 <= r["nrhs"] <= 8 for r in a)


KINDS = [("jacobi", "cg"), ("fd", "cg"), ("fd", "bicgstab"), ("jacobi", "bicgstab")]


@pytest.mark.gpu
@pytest.mark.parametrize("precond,method", KINDS[:3])
def test_result_alone_equals_result_in_the_mix(cuda_ok, precond, method):
    """The target request alone, then among CG / BiCGSTAB, Jacobi / fast-
    diagonalisation requests running concurrently (several right-hand sides
    share one operator): the same solution."""
    from yeti_b200.serve import Server
    clamp = {"w0": (0, 1, 2)}
    target = _request((7, 6, 9), 3, 11, 3)
    others = [_request((5, 9, 4), 2, 21, 2), _request((12, 4, 6), 3, 31, 4),
              _request((4, 4, 4), 2, 41, 1), _request((9, 8, 7), 2, 51, 2),
              _request((6, 11, 5), 3, 61, 3)]
    with Server(max_active=1) as srv:
        x_alone, info_alone = srv.wait(srv.submit(target[0], 1.0, 0.3, clamp, target[1],
                                                  rtol=1e-10, precond=precond, method=method))
    with Server(max_active=16) as srv:
        t_before = [srv.submit(o[0], 1.0, 0.25, clamp, o[1], rtol=1e-10,
                               precond=KINDS[i][0], method=KINDS[i][1])
                    for i, o in enumerate(others[:3])]
        t = srv.submit(target[0], 1.0, 0.3, clamp, target[1], rtol=1e-10, precond=precond,
                       method=method)
        t_after = [srv.submit(o[0], 1.0, 0.35, clamp, o[1], rtol=1e-10,
                              precond=KINDS[(i + 1) % 4][0], method=KINDS[(i + 1) % 4][1])
                   for i, o in enumerate(others[3:])]
        x_mix, info_mix = srv.wait(t)
        for tt in t_before + t_after:
            _, inf = srv.wait(tt)
            assert inf["status"] == 0 and max(inf["rel_residual"]) <= 1e-10
        assert srv.stats()["peak_active"] >= 2   # requests overlapped
    assert info_alone["status"] == 0 and info_mix["status"] == 0
    assert max(info_mix["rel_residual"]) <= 1e-10
    for k in range(3):
        assert _rel(x_mix[k], x_alone[k]) < 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("precond,method", KINDS)
def test_served_solution_matches_one_shot_solver(cuda_ok, precond, method):
    from yeti_b200.serve import Server
    from yeti_b200.wq import WQElasticity
    clamp = {"w0": (0, 1, 2)}
    patch, rhs = _request((8, 7, 6), 3, 5, 2)
    with Server() as srv:
        x, info = srv.wait(srv.submit(patch, 1.0, 0.3, clamp, rhs, rtol=1e-10, precond=precond,
                                      method=method))
    op = WQElasticity(patch, 1.0, 0.3, clamp, precisions="f64")
    for k in range(2):
        xr, st = op.pcg(rhs[k], rtol=1e-10, precond=precond, method=method)
        assert _rel(x[k], xr) < 1e-8
        assert info["iterations"][k] > 0


@pytest.mark.gpu
def test_admission_honours_the_hbm_budget(cuda_ok):
    from yeti_b200.serve import Server
    clamp = {"w0": (0, 1, 2)}
    reqs = [_request((10, 10, 10), 3, 100 + i, 2) for i in range(4)]
    # each request is estimated at about 16.4 MB (two FP64 coefficient
    # copies of 25^3 points, vectors, 4 MB of tables): 24 MiB admits one at
    # a time
    with Server(hbm_budget_bytes=24 << 20, max_active=8) as srv:
        ts = [srv.submit(r[0], 1.0, 0.3, clamp, r[1], rtol=1e-8) for r in reqs]
        infos = [srv.wait(t)[1] for t in ts]
        st = srv.stats()
    assert all(i["status"] == 0 for i in infos)
    assert st["peak_active"] == 1
    # the later requests waited for the earlier ones
    assert infos[-1]["queue_ms"] > 0.0


@pytest.mark.gpu
def test_oversized_request_is_refused(cuda_ok):
    from yeti_b200._lib import YetiError
    from yeti_b200.serve import Server
    patch, rhs = _request((16, 16, 16), 3, 7, 1)
    with Server(hbm_budget_bytes=8 << 20) as srv:
        with pytest.raises(YetiError):
            srv.submit(patch, 1.0, 0.3, {"w0": (0, 1, 2)}, rhs)


@pytest.mark.gpu
def test_fd_bicgstab_converges_where_fd_cg_stalls(cuda_ok):
    """A request of the serving stream (p=2, 4x24x28 elements, Gaussian
    right-hand sides) on which FD-preconditioned CG stalls near 1e-7 (the
    operator is not symmetric; the oracle stalls the same way): the served
    FD-BiCGSTAB solve reaches 1e-8."""
    from yeti_b200.serve import Server, synthetic_requests
    r = synthetic_requests(267, seed=20261203 + 7)[266]
    assert tuple(r["patch"]["nel"]) == (4, 24, 28)
    rhs = np.random.default_rng(r["rhs_seed"]).standard_normal((r["nrhs"], r["ndof"]))
    with Server() as srv:
        x, info = srv.wait(srv.submit(r["patch"], r["E"], r["nu"], r["clamp"], rhs, rtol=1e-8,
                                      maxit=2000, precond="fd", method="bicgstab"))
    assert info["status"] == 0
    assert max(info["rel_residual"][:r["nrhs"]]) <= 1e-8
    assert max(info["iterations"][:r["nrhs"]]) < 200
