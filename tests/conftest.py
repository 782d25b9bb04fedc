import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")

SYSTEM_ARG_NAMES = [
    "activeElement", "nb_data", "COORDS3D", "IEN", "nb_elem_patch", "Nkv",
    "Ukv", "Nijk", "weight", "Jpqr", "ELT_TYPE", "PROPS", "JPROPS",
    "MATERIAL_PROPERTIES", "n_mat_props", "RHO", "TENSOR", "indDLoad",
    "JDLType", "ADLMAG", "load_target_nbelem", "load_additionalInfos",
    "nb_load_additionalInfos", "bc_values", "bc_target", "bc_target_nbelem",
    "ind_dof_free", "nb_dof_free", "MCRD", "NBINT", "NNODE", "nodal_dist",
    "nb_bc", "nb_load", "nb_patch", "nb_elem", "nb_cp", "nb_dof_tot",
]


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
