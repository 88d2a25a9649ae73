import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 and the built CUDA library")


def _has_gpu():
    """A CUDA device is visible to the driver (no torch import needed)."""
    import ctypes
    try:
        cu = ctypes.CDLL("libcuda.so.1")
        if cu.cuInit(0) != 0:
            return False
        n = ctypes.c_int(0)
        return cu.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def reference_src():
    """The reference crate's `src/` directory, named by the environment variable
    PR_REFERENCE_SRC; tests that read the crate's sources skip when it is unset or absent."""
    path = os.environ.get("PR_REFERENCE_SRC", "")
    if not path or not os.path.isdir(path):
        pytest.skip("reference sources not available (set PR_REFERENCE_SRC to the crate's src/)")
    return path


@pytest.fixture(scope="session")
def ctx():
    import poissonreconstruction_b200 as prb
    c = prb.Context(0)
    yield c
    c.close()
