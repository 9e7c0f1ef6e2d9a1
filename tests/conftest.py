import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "toposzp-cuda_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: larger CPU cases")


def pytest_collection_modifyitems(config, items):
    # the no-allocation entry-point test file runs last on purpose
    items.sort(key=lambda it: 1 if "test_zz_" in str(it.fspath) else 0)


@pytest.fixture(scope="session")
def ora():
    import oracle
    oracle.build(ref=True)
    return oracle


@pytest.fixture(scope="session")
def ref(ora):
    if not ora.ref_available():
        pytest.skip("reference library not built (reference sources absent)")
    ora.set_ref_threads(1)
    return ora
