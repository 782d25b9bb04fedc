"""ctypes front-end of oracle/oracle_wq.c: the reference's own (rank-one,
non-sum-factorised) WQ apply algorithm on the host cores.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py): used by tests/ to check it
against the numpy oracle and by bench.py's cpu_baseline / reference arm.
"""
import ctypes
import time

import numpy as np

from . import lib, wq_rules


class ReferenceWQ:
    def __init__(self, patch, E, nu, clamp_faces=None):
        from yeti_b200.patches import free_mask
        L = lib()
        L.oracle_wq_create.restype = ctypes.c_void_p
        # every pointer declared, or ctypes passes the addresses as C ints
        vp = ctypes.c_void_p
        L.oracle_wq_create.argtypes = [vp, vp, vp, vp, vp, ctypes.c_double,
                                       ctypes.c_double, vp]
        L.oracle_wq_apply.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_wq_free.argtypes = [ctypes.c_void_p]
        L.oracle_wq_diag.argtypes = [vp, vp]
        L.oracle_wq_pcg_seconds.restype = ctypes.c_double
        L.oracle_wq_pcg_seconds.argtypes = [vp, vp, vp, ctypes.c_int, vp, vp]
        L.oracle_cg_vector_seconds.restype = ctypes.c_double
        L.oracle_cg_vector_seconds.argtypes = [ctypes.c_int64, ctypes.c_int]
        p, nel = patch["p"], patch["nel"]
        rules = [wq_rules.wq_rule(p[d], nel[d]) for d in range(3)]
        self._keep = []
        ptrs = []
        for d in range(3):
            for k in ("B0", "B1", "W00", "W01", "W10", "W11"):
                a = np.ascontiguousarray(rules[d][k], dtype=np.float64)
                self._keep.append(a)
                ptrs.append(a.ctypes.data)
        arr = (ctypes.c_void_p * 18)(*ptrs)
        n = np.array([p[d] + nel[d] for d in range(3)], dtype=np.int32)
        q = np.array([2 * (p[d] + nel[d]) - 1 for d in range(3)], dtype=np.int32)
        cps = np.ascontiguousarray(patch["cps"].T, dtype=np.float64)   # (ncp, 3)
        w = np.ascontiguousarray(patch["weights"], dtype=np.float64)
        self.mask = free_mask(patch, clamp_faces)
        m8 = np.ascontiguousarray(self.mask.astype(np.uint8))
        self.ndof = 3 * int(np.prod(n))
        self.nfree = int(self.mask.sum())
        self.h = L.oracle_wq_create(n.ctypes.data, q.ctypes.data, arr,
                                    cps.ctypes.data, w.ctypes.data,
                                    ctypes.c_double(E), ctypes.c_double(nu),
                                    m8.ctypes.data)
        self.L = L

    def apply(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty_like(u)
        self.L.oracle_wq_apply(self.h, u.ctypes.data, out.ctypes.data)
        return out

    def diag(self):
        """Diagonal of K (find_physical_diag_3d per diagonal block); clamped
        dofs hold 1."""
        d = np.empty(self.ndof)
        self.L.oracle_wq_diag(self.h, d.ctypes.data)
        return d

    def pcg_seconds(self, b, diag, iters):
        """`iters` consecutive Jacobi-PCG iterations from x = 0 (the loop of
        wq_mf_cg_3d, mf_wq_solver.f90:764-802, with z = r / diag), timed as
        one loop: (seconds per iteration, x, ||r|| / ||b||)."""
        bb = np.ascontiguousarray(b, dtype=np.float64)
        dd = np.ascontiguousarray(diag, dtype=np.float64)
        x = np.empty_like(bb)
        rel = ctypes.c_double(0.0)
        t = self.L.oracle_wq_pcg_seconds(self.h, bb.ctypes.data, dd.ctypes.data, int(iters),
                                         x.ctypes.data, ctypes.byref(rel))
        return t, x, rel.value

    def close(self):
        if self.h:
            self.L.oracle_wq_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def time_reference_apply(patch, E, nu, clamp_faces, n_applies=1):
    """Seconds per apply / per CG-iteration vector work on the host."""
    L = lib()
    L.oracle_wq_threads.restype = ctypes.c_int
    t0 = time.perf_counter()
    op = ReferenceWQ(patch, E, nu, clamp_faces)
    setup = time.perf_counter() - t0
    u = np.random.default_rng(0).standard_normal(op.ndof) * op.mask
    t0 = time.perf_counter()
    for _ in range(n_applies):
        op.apply(u)
    t_apply = (time.perf_counter() - t0) / n_applies
    t_vec = L.oracle_cg_vector_seconds(op.ndof, 5)
    res = {"seconds_per_apply": t_apply, "seconds_per_vector_ops": t_vec,
           "setup_s": setup, "nfree": op.nfree, "ndof": op.ndof,
           "threads": int(L.oracle_wq_threads())}
    op.close()
    return res


def time_reference_cg(patch, E, nu, clamp_faces, iters=10, seed=0):
    """Seconds per Jacobi-PCG iteration of the reference's algorithm on the
    host cores: `iters` consecutive iterations (apply + vector work) timed as
    one loop, on a seeded right-hand side."""
    L = lib()
    L.oracle_wq_threads.restype = ctypes.c_int
    t0 = time.perf_counter()
    op = ReferenceWQ(patch, E, nu, clamp_faces)
    setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    d = op.diag()
    t_diag = time.perf_counter() - t0
    b = np.random.default_rng(seed).standard_normal(op.ndof) * op.mask
    t_it, _, rel = op.pcg_seconds(b, d, iters)
    res = {"seconds_per_iteration": t_it, "iterations_timed": int(iters),
           "rel_residual_after": rel, "setup_s": setup, "diag_s": t_diag,
           "nfree": op.nfree, "ndof": op.ndof, "threads": int(L.oracle_wq_threads())}
    op.close()
    return res
