import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libdimcv.so")


@pytest.fixture(scope="session")
def cuda():
    """GPU tests fail (not skip) without CUDA: a skipped parity test is not a pass."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA is not available; -m gpu tests need a GPU")
    from dimcv_sph_b200 import _lib
    _lib.load()
    return torch.device("cuda:0")
