import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")

from yeti_b200.stiffmtrx_elemstorage import SYSTEM_ARG_NAMES  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_fixture(name):
    """(npz dict, positional argument list of sys_linmat_lindef_static)."""
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    args = [d[k] if d[k].ndim else d[k][()] for k in SYSTEM_ARG_NAMES]
    return d, args


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
