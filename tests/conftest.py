import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a); run with -m gpu")
    config.addinivalue_line("markers", "slow: full-size property checks")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def gpu():
    """The CUDA device for -m gpu tests; fails (not skips) without one, so a
    GPU run never passes silently on a machine without the GPU path."""
    import torch
    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    from tsm_benchmark_b200 import _capi
    _capi.load()
    return torch.device("cuda", 0)
