import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def native_lib():
    from tdp1375_b200 import native
    return native.load()


@pytest.fixture(scope="session")
def gpu_searcher(native_lib):
    """One GPUSortingSearch with two slots on device 0 (queue budget 256 MB, 2M entries)."""
    from tdp1375_b200 import GPUSortingSearch
    g = GPUSortingSearch(1, 2, 256 << 20, 1 << 21)
    yield g
    GPUSortingSearch.destroySlots()


def load_golden(name):
    import json
    with open(os.path.join(ROOT, "tests", "golden", name)) as fh:
        return json.load(fh)
