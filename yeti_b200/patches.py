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


def u1_system_args(patch, E=1.0, nu=0.3, rho=0.0, nbint=None, clamp_u0=False,
                   load_u1=None):
    """The 38 positional arguments of ``sys_linmat_lindef_static`` (the
    order of ``IGAparametrization.get_inputs4system_elemStorage()``,
    IGA_parametrization.py:1705-1716) for a single U1 patch from
    :func:`cube_patch`: every element active, NBINT = (max p + 1)^3 unless
    given.  Without options no loads and no boundary conditions (all dofs
    free).  ``clamp_u0``: the three displacement components of the control
    points on the face u = 0 prescribed to zero; ``load_u1 = (type, mag)``:
    the distributed load 'U2<type>' (face 2, the face u = 1: type 0 normal
    pressure, 1..3 a fixed direction) of magnitude mag on the elements of
    that face.

    IEN lists each element's control points in the reference's descending
    local order: local node (i, j, k) is the control point of tensor index
    (span_u - 1 - i, span_v - 1 - j, span_w - 1 - k), spans 1-based."""
    p, nel = patch["p"], patch["nel"]
    n = [p[d] + nel[d] for d in range(3)]
    kvs = [np.concatenate([np.zeros(p[d] + 1), np.arange(1, nel[d]) / nel[d],
                           np.ones(p[d] + 1)]) for d in range(3)]
    nb_cp = n[0] * n[1] * n[2]
    nb_elem = nel[0] * nel[1] * nel[2]
    nn = (p[0] + 1) * (p[1] + 1) * (p[2] + 1)
    ew, ev, eu = np.meshgrid(np.arange(nel[2]), np.arange(nel[1]),
                             np.arange(nel[0]), indexing="ij")
    nijk = np.stack([eu.ravel() + p[0] + 1, ev.ravel() + p[1] + 1,
                     ew.ravel() + p[2] + 1])           # (3, nb_elem)
    k, j, i = np.meshgrid(np.arange(p[2] + 1), np.arange(p[1] + 1),
                          np.arange(p[0] + 1), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()            # local node order
    iu = nijk[0][:, None] - 1 - i[None, :]
    iv = nijk[1][:, None] - 1 - j[None, :]
    iw = nijk[2][:, None] - 1 - k[None, :]
    cp0 = iu + n[0] * (iv + n[1] * iw)                  # (nb_elem, nn), 0-based
    ien = (cp0 + 1).astype(np.int64).ravel()
    weight = np.asarray(patch["weights"], dtype=np.float64)[cp0].ravel()
    ng = max(p) + 1
    nbint = ng ** 3 if nbint is None else int(nbint)
    ndof = 3 * nb_cp
    if clamp_u0:
        face_cps = (np.arange(n[1] * n[2]) * n[0] + 1).astype(np.int64)   # iu = 0
        bc_values = np.array([[1.0, 2.0, 3.0], [0.0, 0.0, 0.0]])
        bc_target = np.concatenate([face_cps] * 3)
        bc_nb = np.full(3, face_cps.size, dtype=np.int64)
        fixed = np.zeros(ndof, dtype=bool)
        for c in range(3):
            fixed[3 * (face_cps - 1) + c] = True
        free = np.flatnonzero(~fixed) + 1
        ind_dof_free = np.zeros(ndof, dtype=np.int64)   # free dofs first, zeros after
        ind_dof_free[:free.size] = free
        nb_dof_free, nb_bc = int(free.size), 3
    else:
        bc_values = np.zeros((2, 0))
        bc_target = np.zeros(0, dtype=np.int64)
        bc_nb = np.zeros(0, dtype=np.int64)
        ind_dof_free = np.arange(1, ndof + 1, dtype=np.int64)
        nb_dof_free, nb_bc = ndof, 0
    if load_u1 is not None:
        typ, mag = load_u1
        face_el = (np.flatnonzero(eu.ravel() == nel[0] - 1) + 1).astype(np.int64)
        loads = [face_el, np.array([20 + int(typ)], dtype=np.int64),
                 np.array([float(mag)]), np.array([face_el.size], dtype=np.int64),
                 np.zeros(0, dtype=np.float64), np.zeros(1, dtype=np.int64)]
        nb_load = 1
    else:
        loads = [np.zeros(0, dtype=np.int64), np.zeros(0, dtype=np.int64),
                 np.zeros(0, dtype=np.float64), np.zeros(0, dtype=np.int64),
                 np.zeros(0, dtype=np.float64), np.zeros(0, dtype=np.int64)]
        nb_load = 0
    return [
        np.ones(nb_elem, dtype=np.int64),                      # activeElement
        float(nb_elem * (9 * nn * (nn - 1) // 2 + 6 * nn)),    # nb_data
        np.asarray(patch["cps"], dtype=np.float64),            # COORDS3D
        ien,                                                   # IEN
        np.array([nb_elem], dtype=np.int64),                   # nb_elem_patch
        np.array([[len(kv)] for kv in kvs], dtype=np.int64),   # Nkv (3, 1)
        np.concatenate(kvs),                                   # Ukv
        nijk.astype(np.int64),                                 # Nijk
        weight,                                                # weight
        np.array([[p[0]], [p[1]], [p[2]]], dtype=np.int64),    # Jpqr
        np.array("U1"),                                        # ELT_TYPE
        np.array([1.0]), np.array([1], dtype=np.int64),        # PROPS, JPROPS
        np.array([[E], [nu]], dtype=np.float64),               # MATERIAL_PROPERTIES
        np.array([3], dtype=np.int64),                         # n_mat_props
        np.array([rho], dtype=np.float64),                     # RHO
        np.array("/THREED"),                                   # TENSOR
        *loads,   # indDLoad, JDLType, ADLMAG, load_target_nbelem, infos, nb infos
        bc_values,                                             # bc_values
        bc_target,                                             # bc_target
        bc_nb,                                                 # bc_target_nbelem
        ind_dof_free,                                          # ind_dof_free
        nb_dof_free,                                           # nb_dof_free
        3,                                                     # MCRD
        np.array([nbint], dtype=np.int64),                     # NBINT
        np.array([nn], dtype=np.int64),                        # NNODE
        np.zeros((1, nb_cp), dtype=np.float64),                # nodal_dist
        nb_bc, nb_load, 1, nb_elem, nb_cp, ndof,   # nb_bc, nb_load, nb_patch, nb_elem, nb_cp, nb_dof_tot
    ]


def u1_system_args_multi(patches, materials=None, rho=0.0):
    """The 38 arguments of ``sys_linmat_lindef_static`` for several U1
    patches side by side in one model: control points numbered patch after
    patch (no shared control points), elements, knots, IEN, spans and
    weights concatenated in patch order, ``ELT_TYPE`` 'U1U1...', ``TENSOR``
    '/THREED/THREED...', one (E, nu) per patch from ``materials`` (default
    (1, 0.3)) and the Gauss points per element of each patch its own
    (max p + 1)^3."""
    per = [u1_system_args(P) for P in patches]
    npatch = len(per)
    materials = materials or [(1.0, 0.3)] * npatch
    ncps = [int(a[36]) for a in per]
    off = np.cumsum([0] + ncps[:-1])
    nb_cp = int(sum(ncps))
    nb_elem = int(sum(int(a[35]) for a in per))
    nb_data = float(sum(float(a[1]) for a in per))
    coords = np.concatenate([np.asarray(a[2]) for a in per], axis=1)
    ien = np.concatenate([np.asarray(a[3]) + o for a, o in zip(per, off)])
    nkv = np.concatenate([np.asarray(a[5]) for a in per], axis=1)
    ndof = 3 * nb_cp
    return [
        np.ones(nb_elem, dtype=np.int64),
        nb_data,
        coords,
        ien.astype(np.int64),
        np.array([int(a[35]) for a in per], dtype=np.int64),
        nkv.astype(np.int64),
        np.concatenate([np.asarray(a[6]) for a in per]),
        np.concatenate([np.asarray(a[7]) for a in per], axis=1).astype(np.int64),
        np.concatenate([np.asarray(a[8]) for a in per]),
        np.concatenate([np.asarray(a[9]) for a in per], axis=1).astype(np.int64),
        np.array("U1" * npatch),
        np.ones(npatch), np.ones(npatch, dtype=np.int64),
        np.array([[E for E, _ in materials], [nu for _, nu in materials]], dtype=np.float64),
        np.full(npatch, 3, dtype=np.int64),
        np.full(npatch, rho, dtype=np.float64),
        np.array("/THREED" * npatch),
        np.zeros(0, dtype=np.int64), np.zeros(0, dtype=np.int64), np.zeros(0, dtype=np.float64),
        np.zeros(0, dtype=np.int64), np.zeros(0, dtype=np.float64), np.zeros(0, dtype=np.int64),
        np.zeros((2, 0), dtype=np.float64), np.zeros(0, dtype=np.int64), np.zeros(0, dtype=np.int64),
        np.arange(1, ndof + 1, dtype=np.int64),
        ndof,
        3,
        np.concatenate([np.asarray(a[29]) for a in per]).astype(np.int64),
        np.concatenate([np.asarray(a[30]) for a in per]).astype(np.int64),
        np.zeros((1, nb_cp), dtype=np.float64),
        0, 0, npatch, nb_elem, nb_cp, ndof,
    ]


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


def patch_from_iga_model(model, ipatch=0):
    """The WQ description of patch ipatch (0-based: the reference's numpatch
    minus one) of a YETI ``IGAparametrization``, as ``fortran_mf_wq``
    builds it from ``modelIGA`` (``thermoMechaModel.__set_bspline_properties``,
    ``create_model.py:287-354``): degrees from ``_Jpqr``, element counts
    ``_Nkv - (2p + 1)``, knot vectors ``_Ukv`` (uniform and open, the WQ
    rule's hypothesis), control points ``_COORDS`` and weights
    (``_weight``, per element).

    The tensor position (iu, iv, iw) of every control point is read from the
    connectivity, not assumed: YETI's element e with knot spans ``_Nijk[:, e]``
    (1-based) lists its nodes with the u index fastest and every 1-D index
    descending (``shap.f90:91-119``), so node a = i + (p+1)(j + (q+1)k)
    has tensor index (Nijk[0,e]-1-i, Nijk[1,e]-1-j, Nijk[2,e]-1-k).

    Returns (patch, cp_index): the patch dict of ``cube_patch``'s form and,
    per tensor position (u fastest), the 0-based model control point."""
    Jpqr = np.asarray(model._Jpqr).reshape(3, -1)
    Nkv = np.asarray(model._Nkv).reshape(3, -1)
    p = [int(Jpqr[d, ipatch]) for d in range(3)]
    nel = [int(Nkv[d, ipatch]) - (2 * p[d] + 1) for d in range(3)]
    for d in range(3):
        kv = np.asarray(model._Ukv[ipatch][d], dtype=np.float64)
        ref = np.concatenate([np.zeros(p[d] + 1), np.arange(1, nel[d]) / nel[d],
                              np.ones(p[d] + 1)])
        if kv.shape != ref.shape or np.abs(kv - ref).max() > 1e-12:
            raise ValueError(f"patch {ipatch}: knot vector {d} is not uniform and open "
                             "(the weighted-quadrature rules assume it)")
    n = [p[d] + nel[d] for d in range(3)]
    ncp = n[0] * n[1] * n[2]
    nbp = np.asarray(model._elementsByPatch).ravel()
    e0 = int(nbp[:ipatch].sum())
    ien = np.asarray(model._IEN[ipatch]).reshape(int(nbp[ipatch]), -1)
    nijk = np.asarray(model._Nijk).reshape(3, -1)
    cp_index = np.full(ncp, -1, dtype=np.int64)
    weights = np.zeros(ncp)
    a = np.arange(ien.shape[1])
    li = a % (p[0] + 1)
    lj = (a // (p[0] + 1)) % (p[1] + 1)
    lk = a // ((p[0] + 1) * (p[1] + 1))
    for e in range(ien.shape[0]):
        s = nijk[:, e0 + e]
        t = (s[0] - 1 - li) + n[0] * ((s[1] - 1 - lj) + n[1] * (s[2] - 1 - lk))
        cp_index[t] = ien[e] - 1
        weights[t] = np.asarray(model._weight[e0 + e], dtype=np.float64)
    if (cp_index < 0).any() or np.unique(cp_index).size != ncp:
        raise ValueError(f"patch {ipatch}: the connectivity does not cover a tensor grid")
    X = np.asarray(model._COORDS, dtype=np.float64)[:3]
    patch = {"p": tuple(p), "nel": tuple(nel),
             "cps": np.ascontiguousarray(X[:, cp_index]),
             "weights": np.ascontiguousarray(weights)}
    return patch, cp_index


def clamp_faces_from_blocked(blocked):
    """The reference's ``mechablockedboundaries`` ([[u0, u1], [v0, v1],
    [w0, w1]] flags, all three components blocked on a flagged face:
    ``block_boundaries(typeEl='D')``, create_model.py:434-529) as
    clamp_faces."""
    names = (("u0", "u1"), ("v0", "v1"), ("w0", "w1"))
    out = {}
    for d in range(3):
        for s in range(2):
            if blocked[d][s]:
                out[names[d][s]] = (0, 1, 2)
    return out
