"""numpy restatement of the reference's 1-D weighted-quadrature rule.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Follows src/yeti_iga/iga_wq_mf/fsrc/iga_wq_methods.f90 (r = 2, maxrule = 1,
uniform open knot vectors): point positions (wq_get_qp_positions, :38-89),
supports (wq_get_B0_B1_shape, :200-292), exact Gauss integrals and one local
least-squares / minimum-norm solve per test function
(wq_get_basis_weights_generalized, :420-599, with numpy.linalg.lstsq standing
in for LAPACK dgesv/dgels), and the (p+3)-element model copied and rescaled for
larger meshes (wq_get_basis_weights_model, :601-650; wq_get_basis_weights,
:852-1011).  Returns dense (nfun x nqp) matrices.
"""
import numpy as np

SPAN_TOL = 1e-8
TOL = 1e-15


def npts(p, nel):
    return 2 * (p + 2) + 2 * nel - 5


def nodes(nel):
    n = np.array([i / nel for i in range(nel + 1)], dtype=np.float64)
    n[0], n[-1] = 0.0, 1.0
    return n


def knots(p, nd):
    return np.concatenate([np.zeros(p + 1), nd[1:-1], np.ones(p + 1)])


def points(p, nel):
    nd = nodes(nel)
    n = npts(p, nel)
    x = np.zeros(n)

    def linspace(a, b, m):
        h = (b - a) / (m - 1)
        o = a + np.arange(m) * h
        o[0], o[-1] = a, b
        return o

    x[:p + 2] = linspace(nd[0], nd[1], p + 2)
    x[n - (p + 2):] = linspace(nd[nel - 1], nd[nel], p + 2)
    for i in range(1, nel - 1):
        k = (p + 2) + 2 * (i - 1) - 1
        x[k:k + 3] = linspace(nd[i], nd[i + 1], 3)
    return x


def _ders(span, p, u, U):
    """Values and first derivatives of the p+1 B-splines nonzero on 1-based
    knot span `span` (The NURBS Book A2.3, dersbasisfuns.f90:30-131)."""
    ndu = np.zeros((p + 1, p + 1))
    left = np.zeros(p + 2)
    right = np.zeros(p + 2)
    ndu[0, 0] = 1.0
    for j in range(1, p + 1):
        left[j] = u - U[span - j]
        right[j] = U[span + j - 1] - u
        saved = 0.0
        for r in range(j):
            ndu[j, r] = right[r + 1] + left[j - r]
            temp = ndu[r, j - 1] / ndu[j, r]
            ndu[r, j] = saved + right[r + 1] * temp
            saved = left[j - r] * temp
        ndu[j, j] = saved
    N = ndu[:, p].copy()
    dN = np.zeros(p + 1)
    for r in range(p + 1):
        d = 0.0
        if p >= 1:
            if r >= 1:
                d += ndu[r - 1, p - 1] / ndu[p, r - 1]
            if r <= p - 1:
                d -= ndu[r, p - 1] / ndu[p, r]
        dN[r] = d * p
    return N, dN


def basis(p, nel, x):
    """Dense (nfun x len(x)) B-spline values and derivatives (get_basis,
    bspline.f90:200-258, spans found with the reference's 1e-8 tolerance)."""
    nd = nodes(nel)
    U = knots(p, nd)
    nfun = p + nel
    B0 = np.zeros((nfun, len(x)))
    B1 = np.zeros((nfun, len(x)))
    for q, xq in enumerate(x):
        el = 2
        while el < nel + 1 and nd[el - 1] - xq <= SPAN_TOL:
            el += 1
        el -= 1
        ks = p + 2
        while ks < nfun + 1 and U[ks - 1] - xq <= SPAN_TOL:
            ks += 1
        ks -= 1
        N, dN = _ders(ks, p, xq, U)
        B0[el - 1:el + p, q] = N
        B1[el - 1:el + p, q] = dN
    return B0, B1


def supports(p, nel):
    """0-based inclusive (B0 lo, B0 hi, B1 lo, B1 hi) point ranges."""
    n = npts(p, nel)
    nfun = p + nel
    s0 = np.zeros(nel, dtype=int)
    s1 = np.zeros(nel, dtype=int)
    s0[0], s1[0] = 1, p + 2
    s0[nel - 1], s1[nel - 1] = n + 1 - (p + 2), n
    for i in range(1, nel - 1):
        s0[i] = s1[i - 1]
        s1[i] = s0[i] + 2
    out = np.zeros((nfun, 4), dtype=int)
    for i in range(nfun):
        lo = s0[max(0, i - p)]
        hi = s1[min(nel - 1, i)]
        l0, h0, l1, h1 = lo, hi, lo, hi
        if i == 0:
            h0 -= 1
        elif i == nfun - 1:
            l0 += 1
        else:
            h0 -= 1
            l0 += 1
        if i in (0, 1):
            h1 -= 1
        elif i in (nfun - 1, nfun - 2):
            l1 += 1
        else:
            h1 -= 1
            l1 += 1
        out[i] = (l0 - 1, h0 - 1, l1 - 1, h1 - 1)
    return out


def _rules(MB, MI, Mint, sup):
    nrows, nqp = MB.shape
    nfun = MI.shape[1]
    W = np.zeros((nfun, nqp))
    for i in range(nfun):
        rows = np.nonzero(Mint[:, i] > 0)[0]
        fmin, fmax = rows.min(), rows.max()
        lo, hi = sup[i, 0], sup[i, 1]
        A = MB[fmin:fmax + 1, lo:hi + 1]
        b = MI[fmin:fmax + 1, i]
        W[i, lo:hi + 1] = np.linalg.lstsq(A, b, rcond=None)[0]
    return W


def _generalized(p, nel):
    nd = nodes(nel)
    x = points(p, nel)
    xg, wg = np.polynomial.legendre.leggauss(p + 1)
    xc = np.concatenate([0.5 * (xg / nel + nd[i + 1] + nd[i]) for i in range(nel)])
    wc = np.concatenate([0.5 / nel * wg for _ in range(nel)])
    B0c, B1c = basis(p, nel, xc)
    B0, B1 = basis(p, nel, x)
    B0c1, _ = basis(p - 1, nel, xc)
    B0w1, _ = basis(p - 1, nel, x)
    sup = supports(p, nel)
    I0 = (np.abs(B0c) > TOL).astype(int) @ (np.abs(B0c) > TOL).astype(int).T
    I1 = (np.abs(B0c1) > TOL).astype(int) @ (np.abs(B0c) > TOL).astype(int).T
    W00 = _rules(B0, (B0c * wc) @ B0c.T, I0, sup)
    W10 = _rules(B0, (B0c * wc) @ B1c.T, I0, sup)
    W01 = _rules(B0w1, (B0c1 * wc) @ B0c.T, I1, sup)
    W11 = _rules(B0w1, (B0c1 * wc) @ B1c.T, I1, sup)
    return dict(x=x, B0=B0, B1=B1, W00=W00, W01=W01, W10=W10, W11=W11,
                sup=sup)


def wq_rule(p, nel):
    """Dense 1-D WQ rule: dict with x, B0, B1, W00, W01, W10, W11."""
    if nel <= p + 3:
        return _generalized(p, nel)
    nm = p + 3
    M = _generalized(p, nm)
    up, dn = nel / nm, nm / nel
    nfun, nqp = p + nel, npts(p, nel)
    sup = supports(p, nel)
    R = dict(x=points(p, nel), sup=sup)
    for k in ("B0", "B1", "W00", "W01", "W10", "W11"):
        R[k] = np.zeros((nfun, nqp))

    def put(i, j, mi, mj, sgn):
        R["B0"][i, j] = M["B0"][mi, mj]
        R["B1"][i, j] = sgn * M["B1"][mi, mj] * up
        R["W00"][i, j] = M["W00"][mi, mj] * dn
        R["W01"][i, j] = M["W01"][mi, mj] * dn
        R["W10"][i, j] = sgn * M["W10"][mi, mj]
        R["W11"][i, j] = sgn * M["W11"][mi, mj]

    for i in range(p + 1):
        for j in range(sup[i, 2], sup[i, 3] + 1):
            put(i, j, i, j, 1.0)
    mid = p + 1
    msup = M["sup"]
    width = msup[mid, 3] - msup[mid, 2] + 1
    for i in range(p + 1, nfun - p - 1):
        for j in range(width):
            put(i, sup[i, 2] + j, mid, msup[mid, 2] + j, 1.0)
    for i in range(p + 1):
        for j in range(sup[i, 2], sup[i, 3] + 1):
            put(nfun - 1 - i, nqp - 1 - j, i, j, -1.0)
    return R


def exact_integrals(p, nel):
    """Exact 1-D Gram matrices (nfun x nfun): int B_i B_j, int B_i B_j',
    int B_i' B_j, int B_i' B_j' by Gauss quadrature with p+1 points."""
    nd = nodes(nel)
    xg, wg = np.polynomial.legendre.leggauss(p + 1)
    xc = np.concatenate([0.5 * (xg / nel + nd[i + 1] + nd[i]) for i in range(nel)])
    wc = np.concatenate([0.5 / nel * wg for _ in range(nel)])
    B0, B1 = basis(p, nel, xc)
    return {"00": (B0 * wc) @ B0.T, "01": (B0 * wc) @ B1.T,
            "10": (B1 * wc) @ B0.T, "11": (B1 * wc) @ B1.T}
