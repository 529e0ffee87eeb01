import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs liblgv.so kernels)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle  # oracle/oracle.py (test infrastructure)
    oracle.load()
    return oracle


@pytest.fixture(scope="session")
def lgv():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test collected without a CUDA device")
    import langevina_b200 as lgv_pkg
    return lgv_pkg
