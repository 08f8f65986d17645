"""The bounds-checked engine (libpava_gpu_bounds.so, PAVA_BOUNDS_CHECK): the same results as the
ordinary build with no failed index test, and a bad column planted in a caller's CSR is counted
and skipped instead of read.  Runs tests/bounds_check_run.py in a process of its own, where
PAVA_GPU_LIB makes the checked library the one that loads."""
import ctypes
import json
import os
import subprocess
import sys

import pytest

from pava_b200 import _abi
from pava_b200 import build as B

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bounds_checked_build(cuda):
    lib = B.build_bounds()
    env = dict(os.environ, PAVA_GPU_LIB=lib)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "bounds_check_run.py")],
                       capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stdout + r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["library"] == "libpava_gpu_bounds.so" and out["checked"] == 1
    # every form within its bound, no index outside its array
    assert out["max_rel_err_fp64"] <= 1e-12 and out["max_rel_err_fp32c"] <= 1e-9, out
    assert out["failed_tests_clean"] == 0, out
    # the planted column n + 3: caught at the x gather (site 1) with its index, and skipped
    assert out["planted_failed_tests"] >= 1, out
    assert out["planted_site"] == 1 and out["planted_index"] == out["planted_n"] + 3, out
    assert out["planted_row_skipped"] and out["planted_rows_finite"], out


def test_ordinary_build_reports_no_checks(cuda):
    L = _abi.gpu()
    if L.pava_bounds_checked():
        pytest.skip("the checked library is loaded in this process")
    out = (ctypes.c_ulonglong * 3)()
    assert L.pava_bounds_report(out, 0) == _abi.E_UNSUPPORTED_PARAMS
    assert list(out) == [0, 0, 0]
