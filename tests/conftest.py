import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def lib():
    """The product library; on a GPU box it must load (no fallback)."""
    from multilayersolver2024_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def gpu(lib):
    n = lib.mlx_device_count()
    assert n > 0, "GPU test needs a visible sm_100 device"
    return 0


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.load()
    return O
