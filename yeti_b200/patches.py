"""Synthetic single-patch NURBS solids used by the weighted-quadrature path.

A patch is a dict: ``p`` (3 degrees), ``nel`` (3 element counts), ``cps``
(3, ncp) control points and ``weights`` (ncp), with the CP index
``iu + n_u*(iv + n_v*iw)`` and uniform open knot vectors -- the reference's WQ
hypothesis (iga_wq_mf/fsrc/iga_wq_methods.f90:1-10).
"""
import numpy as np


def greville(p, nel):
    """Greville abscissae of the uniform open knot vector (p + nel values)."""
    kv = np.concatenate([np.zeros(p + 1), np.arange(1, nel) / nel,
                         np.ones(p + 1)])
    n = p + nel
    return np.array([kv[i + 1:i + p + 1].mean() for i in range(n)])


def cube_patch(nel, p, size=(1.0, 1.0, 1.0), perturb=0.0, wrange=None,
               seed=0):
    """Block [0,size] meshed with nel[d] uniform elements of degree p[d].

    perturb: interior control points are moved by U(-perturb*h, perturb*h)
    per coordinate (h = element size of that direction); boundary control
    points stay on the faces.  wrange: (lo, hi) draws every weight from
    U(lo, hi); None keeps all weights 1.  Seeded with numpy default_rng(seed).
    """
    nel = tuple(int(n) for n in nel)
    p = tuple(int(q) for q in (p if np.ndim(p) else (p, p, p)))
    rng = np.random.default_rng(seed)
    g = [greville(p[d], nel[d]) * size[d] for d in range(3)]
    n = [p[d] + nel[d] for d in range(3)]
    W, V, U = np.meshgrid(g[2], g[1], g[0], indexing="ij")
    cps = np.stack([U.ravel(), V.ravel(), W.ravel()])   # (3, ncp), u fastest
    if perturb:
        iw, iv, iu = np.meshgrid(np.arange(n[2]), np.arange(n[1]),
                                 np.arange(n[0]), indexing="ij")
        interior = ((iu > 0) & (iu < n[0] - 1) & (iv > 0) & (iv < n[1] - 1) &
                    (iw > 0) & (iw < n[2] - 1)).ravel()
        h = [size[d] / nel[d] for d in range(3)]
        for d in range(3):
            delta = rng.uniform(-perturb * h[d], perturb * h[d], cps.shape[1])
            cps[d] += np.where(interior, delta, 0.0)
    if wrange is None:
        weights = np.ones(cps.shape[1])
    else:
        weights = rng.uniform(wrange[0], wrange[1], cps.shape[1])
    return {"p": p, "nel": nel, "cps": np.ascontiguousarray(cps),
            "weights": np.ascontiguousarray(weights)}


def face_mask(clamp_faces):
    """dirichlet[6*c + f] array from {'u0': comps, 'w1': comps, ...}."""
    names = ["u0", "u1", "v0", "v1", "w0", "w1"]
    m = np.zeros(18, dtype=np.uint8)
    for face, comps in (clamp_faces or {}).items():
        f = names.index(face)
        for c in comps:
            m[6 * c + f] = 1
    return m


def free_mask(patch, clamp_faces):
    """(3*ncp,) 1.0 on free dofs, 0.0 on clamped ones, component-major."""
    n = [patch["p"][d] + patch["nel"][d] for d in range(3)]
    dm = face_mask(clamp_faces)
    iw, iv, iu = np.meshgrid(np.arange(n[2]), np.arange(n[1]),
                             np.arange(n[0]), indexing="ij")
    on = [iu == 0, iu == n[0] - 1, iv == 0, iv == n[1] - 1, iw == 0,
          iw == n[2] - 1]
    out = np.ones((3, n[2], n[1], n[0]))
    for c in range(3):
        for f in range(6):
            if dm[6 * c + f]:
                out[c][on[f]] = 0.0
    return out.ravel()
