import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_addoption(parser):
    parser.addoption("--reference-root", default=os.environ.get("FERRIC_REFERENCE_ROOT"),
                     help="reference checkout whose basis JSONs the oracle pipeline tests read "
                          "(default: $FERRIC_REFERENCE_ROOT; those tests skip without it)")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) device")
    root = config.getoption("--reference-root")
    if root:
        os.environ["FERRIC_REFERENCE_ROOT"] = root


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        return False


@pytest.fixture(scope="session")
def fc():
    """The library bound to cuda:0 (GPU tests only)."""
    if not gpu_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    import ferric_b200._lib as L
    L.init(0)
    return L
