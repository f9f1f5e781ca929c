"""Shared fixtures. Tests marked ``gpu`` need a CUDA device and the built library."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for path in (ROOT, ROOT / "tests"):  # the package, and the shared case modules beside the tests
    if str(path) not in sys.path:
        sys.path.insert(0, str(path))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libmercury_cuda.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def cuda_lib():
    """The built library; on a GPU test this must load and see a device."""
    from mercuda_b200.backend import LIB_PATH, load_library
    if not LIB_PATH.exists():
        from mercuda_b200 import build as B
        B.build()
    lib = load_library()
    if not lib.mercury_cuda_available():
        pytest.fail("libmercury_cuda.so loaded but reports no CUDA device")
    return lib
