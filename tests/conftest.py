import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle.pyoracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.pyoracle import Reference
    try:
        return Reference()
    except OSError as e:
        pytest.skip(str(e))


@pytest.fixture(scope="session")
def lib():
    from fornos_b200 import _lib
    from fornos_b200 import build as B
    B.build()
    return _lib.load()


@pytest.fixture(scope="session")
def ctx(lib):
    if not _has_gpu():
        pytest.skip("no GPU")
    from fornos_b200 import api
    c = api.Context(0)
    yield c
    c.close()
