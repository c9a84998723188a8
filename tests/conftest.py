import os
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
PKG = REPO / "rte-rrtmgp-cpp_b200"
for p in (str(REPO), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built CUDA library")
    config.addinivalue_line("markers", "slow: long-running test")


@pytest.fixture(scope="session")
def tables():
    from rrtmgp_b200 import synthetic as S
    return {"lw": S.make_kdist("lw"), "sw": S.make_kdist("sw"),
            "cloud_lw": S.make_cloud_luts("lw"), "cloud_sw": S.make_cloud_luts("sw")}


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.load()
    return O


@pytest.fixture(scope="session")
def gpu():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from rrtmgp_b200 import _abi
    _abi.load()
    return torch.device("cuda:0")


def rel_err(a, b, floor):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.max(np.abs(a - b) / (np.abs(b) + floor))
