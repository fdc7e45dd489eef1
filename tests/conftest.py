import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a library")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()  # builds oracle/libtg_oracle.so if it is missing
    return oracle


@pytest.fixture(scope="session")
def has_ref(oracle_mod):
    return oracle_mod.ref_lib() is not None


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
