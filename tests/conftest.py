import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build()
    return oracle.Oracle()


@pytest.fixture(scope="session")
def ref_available():
    import oracle
    return oracle.Reference.available()


@pytest.fixture(scope="session")
def nb_lib():
    from mdbas_b200 import nb
    return nb.lib()


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.fail("GPU test run without a CUDA device")
    return 0
