import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))


def golden_system(f):
    """System dictionary of a golden fixture (dense L operators, bcf_exp noise)."""
    from mesohops_b200.bath import bcf_exp
    gw = [[g, w] for g, w in zip(f["G"], f["W"])]
    lops = [np.array(l) for l in f["L"]]
    sysp = {"HAMILTONIAN": np.array(f["H"]), "GW_SYSBATH": gw, "L_HIER": lops,
            "L_NOISE1": lops, "ALPHA_NOISE1": bcf_exp, "PARAM_NOISE1": gw}
    if "LT_L" in f:   # low-temperature corrections
        sysp["L_LT_CORR"] = [np.array(l) for l in f["LT_L"]]
        sysp["PARAM_LT_CORR"] = [complex(c) for c in f["LT_P"]]
    return sysp


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
