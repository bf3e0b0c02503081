import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "df-nvshmem-prototype_b200")
for p in (REPO, os.path.join(PKG, "python")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def repo_root():
    return REPO


@pytest.fixture
def shmem_factory():
    """Starts the library with the given PE count and heap; finalizes after."""
    from nvshmem_b200 import Shmem

    made = []

    def make(npes, heap_bytes, **kw):
        for s in made:
            s.close()
        made.clear()
        s = Shmem(npes, heap_bytes, **kw)
        made.append(s)
        return s

    yield make
    for s in made:
        s.close()
