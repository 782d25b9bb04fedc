"""The C-ABI library: it loads, exports every entry point the header
declares, and fails loudly (an error code, not a crash or a CPU fallback)
where no GPU can be used."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def _declared():
    hdr = open(os.path.join(ROOT, "include", "yeti_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(yeti_\w+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    from yeti_b200 import _lib
    L = _lib.lib()
    names = _declared()
    assert "yeti_assemble_u1_coo" in names and "yeti_wq_pcg" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_library_exports_nothing_undeclared():
    """Only the yeti_* C ABI is visible (built with -fvisibility=hidden)."""
    import subprocess
    from yeti_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH],
                         capture_output=True, text=True).stdout
    syms = {l.split()[-1] for l in out.splitlines() if " T " in l}
    ours = {s for s in syms if s.startswith("yeti_")}
    assert ours == set(_declared())


def test_version_and_launch_counter():
    from yeti_b200 import _lib
    L = _lib.lib()
    assert L.yeti_version().startswith(b"yeti_b200")
    assert isinstance(L.yeti_kernel_launches(), int)


def test_context_creation_reports_errors():
    """Without a usable device the call returns an error code and a message
    (the product path has no CPU fallback)."""
    import torch
    from yeti_b200 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    rc = L.yeti_ctx_create(10_000, 0, ctypes.byref(h))
    assert rc != 0
    assert L.yeti_last_error()
    if not torch.cuda.is_available():
        with pytest.raises(_lib.YetiError):
            _lib.Context(0)


def test_null_arguments_are_rejected():
    from yeti_b200 import _lib
    L = _lib.lib()
    assert L.yeti_assemble_u1_coo(None, None, 0, None, None, None, None, 0) == -1
    assert L.yeti_wq_apply(None, None, None, 0, 0) == -1
    assert L.yeti_wq_pcg(None, None, None, 1e-8, 10, 0, None, 0) == -1
