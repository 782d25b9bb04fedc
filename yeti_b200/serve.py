"""Serving front-end: the persistent WQ solve loop of the C ABI
(yeti_serve_*, include/yeti_b200.h).

    srv = Server(hbm_budget_bytes=8 << 30, max_active=64)
    t = srv.submit(patch, E=1.0, nu=0.3, clamp_faces={"w0": (0, 1, 2)},
                   rhs=np.stack([b1, b2]), rtol=1e-8)
    x, info = srv.wait(t)          # x: (nrhs, ndof)

The engine admits requests in arrival order by slot count and HBM budget,
keeps every admitted operator and its Krylov state on the device, and runs
the solves of all active requests concurrently (CUDA graphs on a stream
pool).  There is no counterpart in the reference, which solves one model per
call.
"""
import ctypes
import threading
import time

import numpy as np

from ._lib import (ServeRequest, ServeResult, YetiError, check, lib, ptr)
from .patches import cube_patch, face_mask
from .wq import _precond_bits


class Server:
    def __init__(self, device=0, hbm_budget_bytes=0, max_active=64):
        h = ctypes.c_void_p()
        check(lib().yeti_serve_open(int(device), int(hbm_budget_bytes),
                                    int(max_active), ctypes.byref(h)),
              "yeti_serve_open")
        self.handle = h
        self._sizes = {}
        self._keep = {}

    def submit(self, patch, E, nu, clamp_faces, rhs, rtol=1e-8, maxit=20000,
               precond="jacobi", method="cg"):
        """Queue a solve of `patch` for each row of rhs ((nrhs, 3*ncp)).
        precond: 'jacobi' or a fast-diagonalisation variant ('fd', ...);
        method: 'cg' or 'bicgstab'.  Returns a ticket at once."""
        p = [int(v) for v in patch["p"]]
        nel = [int(v) for v in patch["nel"]]
        cps = np.ascontiguousarray(np.asarray(patch["cps"], dtype=np.float64).T)
        w = np.ascontiguousarray(patch["weights"], dtype=np.float64)
        rhs = np.ascontiguousarray(np.atleast_2d(rhs), dtype=np.float64)
        ndof = 3 * int(np.prod([p[d] + nel[d] for d in range(3)]))
        if rhs.shape[1] != ndof:
            raise ValueError(f"rhs has {rhs.shape[1]} columns, the patch {ndof} dofs")
        q = ServeRequest()
        q.p[:] = p
        q.nel[:] = nel
        q.cps, q.weights, q.rhs = ptr(cps), ptr(w), ptr(rhs)
        q.E, q.nu = float(E), float(nu)
        q.dirichlet[:] = face_mask(clamp_faces).tolist()
        q.nrhs = rhs.shape[0]
        q.rtol, q.maxit = float(rtol), int(maxit)
        if method not in ("cg", "bicgstab"):
            raise ValueError(f"method {method!r}")
        q.mode = _precond_bits(precond) | (2 if method == "bicgstab" else 0)
        t = ctypes.c_int64()
        check(lib().yeti_serve_submit(self.handle, ctypes.byref(q), ctypes.byref(t)),
              "yeti_serve_submit")
        self._sizes[t.value] = (rhs.shape[0], ndof)
        return t.value

    def _out(self, ticket):
        nrhs, ndof = self._sizes[ticket]
        return np.empty((nrhs, ndof))

    def poll(self, ticket):
        """(x, info) when done, None while pending; raises on failure."""
        x = self._out(ticket)
        res = ServeResult()
        rc = lib().yeti_serve_poll(self.handle, ticket, ptr(x), ctypes.byref(res))
        if rc == 0:
            return None
        self._sizes.pop(ticket, None)
        if rc < 0:
            check(rc, "yeti_serve_poll")
        return x, res.as_dict()

    def wait(self, ticket, timeout_ms=-1.0):
        x = self._out(ticket)
        res = ServeResult()
        rc = lib().yeti_serve_wait(self.handle, ticket, float(timeout_ms), ptr(x),
                                   ctypes.byref(res))
        if rc == -5:   # timed out, still pending
            check(rc, "yeti_serve_wait")
        self._sizes.pop(ticket, None)
        if rc < 0:
            check(rc, "yeti_serve_wait")
        return x, res.as_dict()

    def stats(self):
        done, queued = ctypes.c_int64(), ctypes.c_int64()
        active, peak = ctypes.c_int32(), ctypes.c_int32()
        committed = ctypes.c_size_t()
        check(lib().yeti_serve_stats(self.handle, ctypes.byref(done), ctypes.byref(queued),
                                     ctypes.byref(active), ctypes.byref(peak),
                                     ctypes.byref(committed)), "yeti_serve_stats")
        t = [ctypes.c_double() for _ in range(3)]
        check(lib().yeti_serve_times(self.handle, *[ctypes.byref(v) for v in t]),
              "yeti_serve_times")
        return {"done": done.value, "queued": queued.value, "active": active.value,
                "peak_active": peak.value, "committed_bytes": committed.value,
                "setup_ms": t[0].value, "retire_ms": t[1].value, "poll_ms": t[2].value}

    def close(self):
        if getattr(self, "handle", None):
            lib().yeti_serve_close(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def synthetic_requests(n, seed, p_choices=(2, 3), nel_range=(4, 32),
                       perturb=0.15, wrange=(0.9, 1.1), nu_range=(0.2, 0.4),
                       nrhs_range=(1, 8)):
    """The serving workload: cube-like NURBS patches with p drawn from
    p_choices, element counts per direction uniform in nel_range, interior
    control points perturbed +-perturb*h, weights U(wrange), E = 1, nu
    U(nu_range), clamped at w = 0, and nrhs U(nrhs_range) Gaussian right-hand
    sides.  Seeded; returns a list of dicts."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        p = int(rng.choice(p_choices))
        nel = tuple(int(v) for v in rng.integers(nel_range[0], nel_range[1] + 1, 3))
        patch = cube_patch(nel, p, perturb=perturb, wrange=wrange,
                           seed=int(rng.integers(1 << 31)))
        ndof = 3 * int(np.prod([p + v for v in nel]))
        nrhs = int(rng.integers(nrhs_range[0], nrhs_range[1] + 1))
        out.append({"patch": patch, "E": 1.0, "nu": float(rng.uniform(*nu_range)),
                    "clamp": {"w0": (0, 1, 2)}, "nrhs": nrhs, "ndof": ndof,
                    "rhs_seed": int(rng.integers(1 << 31))})
    return out


def run_stream(server, requests, rate_per_s, seed, rtol=1e-8, precond="jacobi",
               method="cg"):
    """Submit `requests` with Poisson arrivals at rate_per_s (seeded) and
    collect every result.  Returns per-request latencies (ms), the wall time
    from the first submission to the last result (s), and the solved DOF
    (free-or-not dofs x right-hand sides) summed over requests."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, len(requests))
    arrivals = np.cumsum(gaps) - gaps[0]
    tickets = [None] * len(requests)
    results = [None] * len(requests)
    errors = []

    def collector():
        for i in range(len(requests)):
            while tickets[i] is None:
                time.sleep(1e-4)
            try:
                results[i] = server.wait(tickets[i])[1]
            except YetiError as e:   # recorded, reported by the caller
                errors.append((i, str(e)))

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    t0 = time.perf_counter()
    for i, r in enumerate(requests):
        delay = arrivals[i] - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        rhs = np.random.default_rng(r["rhs_seed"]).standard_normal((r["nrhs"], r["ndof"]))
        tickets[i] = server.submit(r["patch"], r["E"], r["nu"], r["clamp"], rhs, rtol=rtol,
                                   precond=precond, method=method)
    th.join()
    wall = time.perf_counter() - t0
    lat = np.array([res["total_ms"] for res in results if res is not None])
    dofs = sum(r["ndof"] * r["nrhs"] for r, res in zip(requests, results) if res is not None)
    return {"latency_ms": lat, "wall_s": wall, "solved_dofs": dofs, "errors": errors,
            "results": results, "offered_s": float(arrivals[-1])}
