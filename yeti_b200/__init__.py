"""yeti_b200: B200-native (sm_100a) implementation of YETI's U1 solid NURBS
path -- Gauss-quadrature element stiffness + COO assembly, the weighted-
quadrature matrix-free operator inside PCG, and the adjoint compliance shape
gradient -- behind a C ABI (include/yeti_b200.h, libyeti_b200.so).

Python entry points mirror the reference's:
  yeti_b200.stiffmtrx_elemstorage.sys_linmat_lindef_static   (f2py twin)
  yeti_b200.wq.WQElasticity   (fortran_mf_wq.eval_Ku / mf_conj_grad twin)
  yeti_b200.gradient.gradlinelastwork_an  (gradadjointwork twin)
"""
from ._lib import Context, YetiError, default_context, lib  # noqa: F401

__version__ = "0.1.0"
