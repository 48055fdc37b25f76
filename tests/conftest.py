import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def tables():
    t = np.load(os.path.join(GOLDEN, "reference_tables.npz"))
    return {k: t[k] for k in t.files}


@pytest.fixture(scope="session")
def po():
    import pyoracle
    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def ops(po, tables):
    return po.Ops.from_tables(tables)


def _has_gpu():
    try:
        from atlas12_b200 import _lib
        return _lib.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_ctx():
    if not _has_gpu():
        pytest.skip("no CUDA device")
    from atlas12_b200 import _lib
    ctx = _lib.Context(0, _lib.PREC_MIXED)
    yield ctx
    ctx.close()
