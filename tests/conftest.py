import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")
    so = os.path.join(ROOT, "oracle", "liblzk_oracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)


@pytest.fixture(scope="session")
def orc():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle import Ref, have_ref
    if not have_ref():
        pytest.skip("oracle/_ref/libref.so (reference host arithmetic) not built here")
    return Ref()


@pytest.fixture()
def rng_state():
    return np.array([0x5EED], np.uint64)


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import liblightzk_b200
    liblightzk_b200.lib()  # raises if the CUDA library is not built
    return torch.device("cuda:0")
