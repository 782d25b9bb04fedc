"""ctypes binding of libyeti_b200.so (the C ABI declared in include/yeti_b200.h).

The library is loaded from the package directory.  There is no fallback: if
the shared object is missing or a CUDA device cannot be used, the calls raise.
"""
import ctypes
import os
import threading

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libyeti_b200.so")

YETI_OK = 0
ERRORS = {-1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "EUNSUPPORTED",
          -5: "ETIMEDOUT", -6: "EBREAKDOWN", -7: "ENUMERIC", -8: "ENOTCONV"}
MEM_HOST, MEM_DEVICE = 0, 1
PREC_F64, PREC_F32 = 0, 1
STIFF_PAIRS, STIFF_SUMFACT = 0, 1

_lib = None
_lock = threading.Lock()


class YetiError(RuntimeError):
    def __init__(self, code, where, msg):
        self.code = code
        super().__init__(f"{where} failed with {ERRORS.get(code, code)}: {msg}")


c_i64 = ctypes.c_int64
c_p = ctypes.c_void_p


class U1Model(ctypes.Structure):
    _fields_ = [
        ("nb_patch", c_i64), ("nb_elem", c_i64), ("nb_cp", c_i64),
        ("coords", c_p), ("ien", c_p), ("nb_elem_patch", c_p), ("nkv", c_p),
        ("ukv", c_p), ("nijk", c_p), ("weight", c_p), ("jpqr", c_p),
        ("nnode", c_p), ("nbint", c_p), ("is_u1", c_p), ("matprops", c_p),
        ("rho", c_p), ("active", c_p), ("nb_load", c_i64), ("inddload", c_p),
        ("jdltype", c_p), ("adlmag", c_p), ("load_target_nbelem", c_p),
        ("load_addinfos", c_p), ("len_load_addinfos", c_i64),
        ("nb_load_addinfos", c_p), ("nb_n_dist", c_i64), ("nodal_dist", c_p),
    ]


class CGStats(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int32), ("outer_iterations", ctypes.c_int32),
        ("fp64_applies", ctypes.c_int32), ("fp32_applies", ctypes.c_int32),
        ("rel_residual", ctypes.c_double), ("rel_residual_inf", ctypes.c_double),
        ("solve_ms", ctypes.c_double), ("status", ctypes.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServeRequest(ctypes.Structure):
    _fields_ = [
        ("p", ctypes.c_int32 * 3), ("nel", ctypes.c_int32 * 3),
        ("cps", c_p), ("weights", c_p), ("E", ctypes.c_double),
        ("nu", ctypes.c_double), ("dirichlet", ctypes.c_uint8 * 18),
        ("nrhs", ctypes.c_int32), ("rhs", c_p), ("rtol", ctypes.c_double),
        ("maxit", ctypes.c_int32), ("mode", ctypes.c_int32),
    ]


class ServeResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32), ("nrhs", ctypes.c_int32),
        ("ndof", c_i64), ("iterations", ctypes.c_int32 * 8),
        ("rel_residual", ctypes.c_double * 8), ("queue_ms", ctypes.c_double),
        ("solve_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
    ]

    def as_dict(self):
        n = self.nrhs
        return {"status": self.status, "ndof": self.ndof,
                "iterations": list(self.iterations[:n]),
                "rel_residual": list(self.rel_residual[:n]),
                "queue_ms": self.queue_ms, "solve_ms": self.solve_ms,
                "total_ms": self.total_ms}


def _declare(lib):
    vp, i32, i64, dbl = c_p, ctypes.c_int, c_i64, ctypes.c_double
    sig = {
        "yeti_last_error": (ctypes.c_char_p, []),
        "yeti_version": (ctypes.c_char_p, []),
        "yeti_kernel_launches": (ctypes.c_uint64, []),
        "yeti_ctx_create": (i32, [i32, ctypes.c_size_t, ctypes.POINTER(vp)]),
        "yeti_ctx_destroy": (i32, [vp]),
        "yeti_ctx_set_stream": (i32, [vp, vp]),
        "yeti_ctx_synchronize": (i32, [vp]),
        "yeti_ctx_bytes_in_use": (ctypes.c_size_t, [vp]),
        "yeti_ctx_set_timing": (i32, [vp, i32]),
        "yeti_ctx_kernel_ms": (ctypes.c_double, [vp, ctypes.c_char_p]),
        "yeti_serve_open": (i32, [i32, ctypes.c_size_t, i32, ctypes.POINTER(vp)]),
        "yeti_serve_submit": (i32, [vp, ctypes.POINTER(ServeRequest), ctypes.POINTER(i64)]),
        "yeti_serve_poll": (i32, [vp, i64, vp, ctypes.POINTER(ServeResult)]),
        "yeti_serve_wait": (i32, [vp, i64, dbl, vp, ctypes.POINTER(ServeResult)]),
        "yeti_serve_stats": (i32, [vp, vp, vp, vp, vp, vp]),
        "yeti_serve_times": (i32, [vp, vp, vp, vp]),
        "yeti_serve_close": (i32, [vp]),
        "yeti_assemble_u1_coo": (i32, [vp, ctypes.POINTER(U1Model), i64, vp,
                                       vp, vp, vp, i32]),
        "yeti_assemble_u1_coo_ex": (i32, [vp, ctypes.POINTER(U1Model), i64, vp,
                                          vp, vp, vp, i32, i32]),
        "yeti_wq_setup": (i32, [vp, vp, vp, vp, vp, dbl, dbl, vp, i32,
                                ctypes.POINTER(vp)]),
        "yeti_wq_destroy": (i32, [vp]),
        "yeti_wq_info": (i32, [vp, vp, vp, vp, vp, vp]),
        "yeti_wq_apply": (i32, [vp, vp, vp, i32, i32]),
        "yeti_wq_apply_static": (i32, [vp, vp, vp, i32]),
        "yeti_wq_set_wait_limit": (i32, [vp, i32]),
        "yeti_wq_diag": (i32, [vp, vp, i32]),
        "yeti_wq_body_force": (i32, [vp, vp, vp, i32]),
        "yeti_wq_pcg": (i32, [vp, vp, vp, dbl, i32, i32,
                              ctypes.POINTER(CGStats), i32]),
        "yeti_wq_pcg_history": (i32, [vp, vp, vp, dbl, i32, i32, vp, vp, vp,
                                      ctypes.POINTER(CGStats), i32]),
        "yeti_wq_fd_apply": (i32, [vp, vp, vp, i32, i32, i32]),
        "yeti_grad_lin_elast_work": (i32, [vp, ctypes.POINTER(U1Model), vp,
                                           vp, i64, i32, i32, i32, vp, vp,
                                           i32]),
        "yeti_volume_u1": (i32, [vp, ctypes.POINTER(U1Model), vp, vp, i32]),
        "yeti_assemble_u1_mass_coo": (i32, [vp, ctypes.POINTER(U1Model), i64, vp, vp,
                                            vp, i32]),
    }
    for name, (res, args) in sig.items():
        if hasattr(lib, name):
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args


def lib():
    """Load libyeti_b200.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with "
                    "`python -m yeti_b200.build` (nvcc, sm_100a)")
            _lib = ctypes.CDLL(LIB_PATH)
            _declare(_lib)
    return _lib


def check(rc, where):
    if rc != YETI_OK:
        msg = lib().yeti_last_error().decode(errors="replace")
        raise YetiError(rc, where, msg)


def exported_symbols():
    """Names of the yeti_* functions declared in include/yeti_b200.h."""
    hdr = os.path.join(os.path.dirname(_PKG), "include", "yeti_b200.h")
    import re
    names = re.findall(r"^\w[\w\s\*]*?\b(yeti_\w+)\s*\(", open(hdr).read(),
                       flags=re.M)
    return sorted(set(names))


def ptr(a):
    """Raw data pointer of a numpy array or a torch tensor."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


# cudaStreamLegacy: the handle of the legacy default stream (a NULL stream
# argument to yeti_ctx_set_stream selects the context's own stream instead).
CUDA_STREAM_LEGACY = 0x1


class Context:
    """A yeti_ctx on one CUDA device (owns a stream unless one is set)."""

    def __init__(self, device=0, hbm_budget_bytes=0):
        h = c_p()
        check(lib().yeti_ctx_create(int(device), int(hbm_budget_bytes),
                                    ctypes.byref(h)), "yeti_ctx_create")
        self.handle = h
        self.device = int(device)

    def set_stream(self, stream):
        """stream: a torch.cuda.Stream, a raw cudaStream_t int, or None."""
        raw = None
        if stream is not None:
            raw = getattr(stream, "cuda_stream", stream)
            if not raw:
                raw = CUDA_STREAM_LEGACY   # torch's default stream has handle 0
        check(lib().yeti_ctx_set_stream(self.handle, raw), "yeti_ctx_set_stream")

    def synchronize(self):
        check(lib().yeti_ctx_synchronize(self.handle), "yeti_ctx_synchronize")

    def bytes_in_use(self):
        return int(lib().yeti_ctx_bytes_in_use(self.handle))

    def set_timing(self, on=True):
        """Sum the device time of the element kernels per name (CUDA events
        on the context's stream); clears the sums."""
        check(lib().yeti_ctx_set_timing(self.handle, int(bool(on))), "yeti_ctx_set_timing")

    def kernel_ms(self, kernel):
        """Summed device ms of `kernel` since set_timing(); None if none."""
        v = float(lib().yeti_ctx_kernel_ms(self.handle, kernel.encode()))
        return None if v < 0 else v

    def close(self):
        if getattr(self, "handle", None):
            lib().yeti_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default = {}


def default_context(device=None):
    """Process-wide context per device (created on first use)."""
    if device is None:
        try:
            import torch
            device = torch.cuda.current_device() if torch.cuda.is_available() else 0
        except Exception:
            device = 0
    with _lock:
        ctx = _default.get(device)
    if ctx is None:
        ctx = Context(device)
        with _lock:
            _default[device] = ctx
    return ctx
