"""Generate golden 1-D weighted-quadrature rules from the reference's own
Python restatement of the WQ rule.

The reference computes its WQ rules in Fortran (iga_wq_mf/fsrc/
iga_wq_methods.f90:12-1011, not buildable here) and ships a pure-Python twin,
``iga_wq_mf/ThermoMechaIGA/pysrc/lib/base_functions.py:308-670``
(``wq_find_basis_weights_opt``).  That module imports two things that are not
installed here:

* ``geomdl.helpers`` (NURBS-Python; the reference pins no version): only
  ``find_span_linear`` and ``basis_function_ders`` are used.  They are
  restated below from their published algorithms (The NURBS Book A2.1 with a
  linear search, and A2.3).
* ``iga_wq_mf.basis_weights`` (the f2py module): only used by
  ``eval_basis_fortran``, which the rule does not call; stubbed.

Writes tests/golden/wq_rules.npz with, for each (p, nel), the dense
(nfun x nqp) matrices B0, B1, W00, W01, W10, W11 and the point positions.
Usage:  python tests/golden/make_wq_golden.py
"""
import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = "src/yeti_iga/iga_wq_mf/ThermoMechaIGA/pysrc/lib"


def reference_root():
    """Root of the reference source tree, from $YETI_REFERENCE."""
    ref = os.environ.get("YETI_REFERENCE")
    if not ref or not os.path.isdir(os.path.join(ref, LIB)):
        raise SystemExit("set YETI_REFERENCE to the root of the reference source tree")
    return ref
CASES = [(2, 2), (2, 3), (2, 5), (2, 8), (3, 2), (3, 4), (3, 6), (3, 9),
         (4, 3), (4, 7), (4, 10)]


def find_span_linear(degree, knot_vector, num_ctrlpts, knot, **_):
    span = degree + 1
    while span < num_ctrlpts and knot_vector[span] <= knot:
        span += 1
    return span - 1


def basis_function_ders(degree, knot_vector, span, knot, order):
    """Values and derivatives up to `order` of the degree+1 nonzero
    B-splines on `span` (0-based) at `knot` (The NURBS Book A2.3)."""
    p = degree
    U = knot_vector
    ndu = [[1.0] * (p + 1) for _ in range(p + 1)]
    left = [1.0] * (p + 1)
    right = [1.0] * (p + 1)
    for j in range(1, p + 1):
        left[j] = knot - U[span + 1 - j]
        right[j] = U[span + j] - knot
        saved = 0.0
        for r in range(j):
            ndu[j][r] = right[r + 1] + left[j - r]
            temp = ndu[r][j - 1] / ndu[j][r]
            ndu[r][j] = saved + right[r + 1] * temp
            saved = left[j - r] * temp
        ndu[j][j] = saved
    ders = [[0.0] * (p + 1) for _ in range(order + 1)]
    for j in range(p + 1):
        ders[0][j] = ndu[j][p]
    a = [[1.0] * (p + 1) for _ in range(2)]
    for r in range(p + 1):
        s1, s2 = 0, 1
        a[0][0] = 1.0
        for k in range(1, order + 1):
            d = 0.0
            rk, pk = r - k, p - k
            if r >= k:
                a[s2][0] = a[s1][0] / ndu[pk + 1][rk]
                d = a[s2][0] * ndu[rk][pk]
            j1 = 1 if rk >= -1 else -rk
            j2 = k - 1 if r - 1 <= pk else p - r
            for j in range(j1, j2 + 1):
                a[s2][j] = (a[s1][j] - a[s1][j - 1]) / ndu[pk + 1][rk + j]
                d += a[s2][j] * ndu[rk + j][pk]
            if r <= pk:
                a[s2][k] = -a[s1][k - 1] / ndu[pk + 1][r]
                d += a[s2][k] * ndu[r][pk]
            ders[k][r] = d
            s1, s2 = s2, s1
    r = p
    for k in range(1, order + 1):
        for j in range(p + 1):
            ders[k][j] *= r
        r *= (p - k)
    return ders


def load_base_functions():
    geomdl = types.ModuleType("geomdl")
    helpers = types.ModuleType("geomdl.helpers")
    helpers.find_span_linear = find_span_linear
    helpers.basis_function_ders = basis_function_ders
    geomdl.helpers = helpers
    sys.modules["geomdl"] = geomdl
    sys.modules["geomdl.helpers"] = helpers
    wq = types.ModuleType("iga_wq_mf")
    wq.basis_weights = types.ModuleType("iga_wq_mf.basis_weights")
    sys.modules["iga_wq_mf"] = wq
    sys.modules["iga_wq_mf.basis_weights"] = wq.basis_weights
    base = os.path.join(reference_root(), LIB, "base_functions.py")
    spec = importlib.util.spec_from_file_location("ref_base_functions", base)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main():
    bf = load_base_functions()
    out = {}
    for p, nel in CASES:
        kv = bf.create_knotvector(p, nel)
        xwq, B0, B1, W00, W01, W10, W11 = bf.wq_find_basis_weights_opt(p, kv, 2)
        tag = f"p{p}_n{nel}"
        out[f"{tag}_x"] = np.asarray(xwq, dtype=np.float64)
        for name, m in (("B0", B0), ("B1", B1), ("W00", W00), ("W01", W01),
                        ("W10", W10), ("W11", W11)):
            out[f"{tag}_{name}"] = np.asarray(m.toarray(), dtype=np.float64)
        print(tag, out[f"{tag}_B0"].shape)
    np.savez_compressed(os.path.join(HERE, "wq_rules.npz"), **out)


if __name__ == "__main__":
    main()
