import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_built():
    from pava_b200 import build as B
    B.build()
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all"], check=True)


_ensure_built()


@pytest.fixture(autouse=True)
def _bounds_report(request):
    """With a bounds-checked engine loaded (PAVA_GPU_LIB=.../libpava_gpu_bounds.so), every GPU
    test must leave the error word at zero: no kernel met an index outside its arrays."""
    yield
    if "cuda" not in request.fixturenames:
        return
    import ctypes
    from pava_b200 import _abi
    L = _abi.gpu()
    if not L.pava_bounds_checked():
        return
    out = (ctypes.c_ulonglong * 3)()
    _abi.check(L.pava_bounds_report(out, 1))
    assert out[0] == 0, (f"bounds check: {out[0]} failed index tests, the first at site "
                         f"{out[1]} with index {out[2]}")


@pytest.fixture(autouse=True)
def _wait_report(request):
    """Every GPU test must leave the bounded-wait word at zero: no kernel gave up waiting on
    its bulk copies (a wait that gives up ends the kernel early with wrong rows)."""
    yield
    if "cuda" not in request.fixturenames:
        return
    import ctypes
    from pava_b200 import _abi
    out = (ctypes.c_ulonglong * 2)()
    st = _abi.gpu().pava_wait_report(out, 1)
    assert st == 0 and out[0] == 0, (f"{out[0]} bounded waits gave up, the first at site "
                                      f"{out[1]}")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pava_b200 import _abi
    _abi.check(_abi.gpu().pava_init(0))
    return torch
