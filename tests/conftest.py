import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def oracle_kind():
    """The strongest oracle present: the reference's own kernels, else the restatement."""
    import oracle
    if os.path.exists(oracle.lib_path("ref")):
        return "ref"
    if not os.path.exists(oracle.lib_path("restate")):
        oracle.build(ref=False)
    return "restate"


@pytest.fixture(scope="session")
def native_lib():
    from camr_b200 import build, native
    if not os.path.exists(native.LIB_PATH):
        build.build()
    return native.lib()
