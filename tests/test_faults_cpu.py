"""Host-side fault injection: damaged inputs and absurd sizes give the documented status
codes, with a message, and never exit or abort (the reference's loader calls exit(1),
utils/basicMatrix.cpp:66-70, and its engines print "-1 -1", main.cpp:309,570).  No GPU: every
failure here is caught before a device call."""
import ctypes

import numpy as np
import pytest

from pava_b200 import _abi
from pava_b200 import matrices as M

GOOD = "%%MatrixMarket matrix coordinate real general\n% comment\n4 5 3\n1 1 1.5\n2 3 -2\n4 5 7\n"


def _read(path):
    H = _abi.host()
    m, n, kind, sym = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    nz = ctypes.c_longlong()
    st = H.pava_mtx_info(str(path).encode(), ctypes.byref(m), ctypes.byref(n), ctypes.byref(nz),
                         ctypes.byref(kind), ctypes.byref(sym))
    if st != 0:
        return st, None
    cap = max(nz.value, 1)
    r, c, v = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap)
    got = ctypes.c_longlong()
    st = H.pava_mtx_read(str(path).encode(), r.ctypes.data, c.ctypes.data, v.ctypes.data,
                         ctypes.byref(got))
    return st, got.value


def test_mtx_good_file_reads(tmp_path):
    p = tmp_path / "good.mtx"
    p.write_text(GOOD)
    assert _read(p) == (0, 3)


@pytest.mark.parametrize("text,status", [
    (GOOD.rsplit("\n", 2)[0] + "\n", _abi.E_CONVERT_FAILED),          # truncated: 2 of 3 entries
    ("%%MatrixMarket matrix coordinate real general\n4 5 3\n", _abi.E_CONVERT_FAILED),  # no entries
    ("%%MatrixMarket matrix coordinate real general\n", _abi.E_CONVERT_FAILED),  # no size line
    ("", _abi.E_CONVERT_FAILED),                                        # empty file
    ("%%NotMatrixMarket matrix coordinate real general\n1 1 1\n1 1 1\n", _abi.E_CONVERT_FAILED),
    ("%%MatrixMarket matrix array real general\n1 1\n1\n", _abi.E_CONVERT_FAILED),  # dense
    ("%%MatrixMarket matrix coordinate real general\n4 5 1\n5 1 1.0\n", _abi.E_INVALID_CSR),
    ("%%MatrixMarket matrix coordinate real general\n4 5 1\n0 1 1.0\n", _abi.E_INVALID_CSR),
    ("%%MatrixMarket matrix coordinate real general\n4 5 1\n1 6 1.0\n", _abi.E_INVALID_CSR),
    ("%%MatrixMarket matrix coordinate real general\n4 5 1\n1 x 1.0\n", _abi.E_INVALID_CSR),
    ("%%MatrixMarket matrix coordinate real general\n3000000000 5 1\n1 1 1.0\n",
     _abi.E_TOO_LARGE),
], ids=["truncated", "no_entries", "no_size_line", "empty", "bad_banner", "dense_array",
        "row_past_m", "row_zero", "col_past_n", "garbled_entry", "rows_past_int32"])
def test_mtx_damaged_files(tmp_path, text, status):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    st, _ = _read(p)
    assert st == status


def test_mtx_missing_file(tmp_path):
    st, _ = _read(tmp_path / "absent.mtx")
    assert st == _abi.E_INVALID_ARG


def test_coo_to_csr_rejects_bad_entries():
    H = _abi.host()
    r = np.array([0, 3], np.int32)
    c = np.array([0, 1], np.int32)
    v = np.ones(2)
    rp, ci, vv = np.zeros(4, np.int32), np.zeros(2, np.int32), np.zeros(2)
    assert H.pava_coo_to_csr(3, 2, 2, r.ctypes.data, c.ctypes.data, v.ctypes.data,
                             rp.ctypes.data, ci.ctypes.data, vv.ctypes.data) == _abi.E_INVALID_CSR
    assert H.pava_coo_to_csr(3, 2, -1, r.ctypes.data, c.ctypes.data, v.ctypes.data,
                             rp.ctypes.data, ci.ctypes.data, vv.ctypes.data) == _abi.E_INVALID_ARG


def _csr(m, n, nnz, arrays=True):
    A = _abi.PavaCsr()
    A.m, A.n, A.nnz = m, n, nnz
    keep = (np.zeros(4, np.int32), np.zeros(4, np.int32), np.zeros(4))
    if arrays:
        A.row_ptr, A.col_idx, A.vals = (a.ctypes.data for a in keep)
    A.on_device = 0
    return A, keep


def _create(A, fmt, **opts):
    o = _abi.PavaOpts()
    for k, v in opts.items():
        setattr(o, k, v)
    h = ctypes.c_void_p()
    st = _abi.gpu().pava_create(ctypes.byref(A), fmt, ctypes.byref(o), None, ctypes.byref(h))
    assert not h.value  # nothing handed out on failure
    return st, _abi.gpu().pava_last_error().decode()


@pytest.mark.parametrize("fmt", [_abi.FORMAT_CVR, _abi.FORMAT_CSR5])
def test_create_absurd_nnz_too_large_without_reading_arrays(fmt):
    # the arrays are 4 entries long: the size check must come before any of them is read
    A, keep = _csr(1000, 1000, 2**31 - 100)
    st, msg = _create(A, fmt)
    assert st == _abi.E_TOO_LARGE and "int32" in msg


def test_create_rows_at_int32_limit():
    A, keep = _csr(2**31 - 1, 10, 0)
    st, msg = _create(A, _abi.FORMAT_CSR)
    assert st == _abi.E_TOO_LARGE and msg


@pytest.mark.parametrize("case,status", [
    ("negative_m", _abi.E_INVALID_ARG), ("negative_nnz", _abi.E_INVALID_ARG),
    ("null_arrays", _abi.E_INVALID_ARG), ("unknown_format", _abi.E_UNKNOWN_FORMAT),
    ("unknown_precision", _abi.E_UNSUPPORTED_VALUE_TYPE),
    ("unknown_index_mode", _abi.E_UNSUPPORTED_PARAMS)])
def test_create_bad_arguments(case, status):
    A, keep = _csr(3, 3, 2)
    fmt, opts = _abi.FORMAT_CVR, {}
    if case == "negative_m":
        A.m = -1
    elif case == "negative_nnz":
        A.nnz = -5
    elif case == "null_arrays":
        A.col_idx = None
    elif case == "unknown_format":
        fmt = 7
    elif case == "unknown_precision":
        opts = dict(precision=9)
    else:
        opts = dict(index_mode=5)
    st, msg = _create(A, fmt, **opts)
    assert st == status and msg


def test_create_null_out_and_matrix():
    L = _abi.gpu()
    A, keep = _csr(3, 3, 2)
    assert L.pava_create(ctypes.byref(A), _abi.FORMAT_CVR, None, None, None) == _abi.E_INVALID_ARG
    h = ctypes.c_void_p()
    assert L.pava_create(None, _abi.FORMAT_CVR, None, None, ctypes.byref(h)) == _abi.E_INVALID_ARG


def test_memory_limit_setting_round_trips():
    L = _abi.gpu()
    old = L.pava_get_device_memory_limit()
    try:
        assert L.pava_set_device_memory_limit(12345) == 0
        assert L.pava_get_device_memory_limit() == 12345
    finally:
        L.pava_set_device_memory_limit(old)
    assert L.pava_get_device_memory_limit() == old


def test_noalloc_too_large_refused_before_any_device_call():
    L = _abi.gpu()
    st = L.pava_spmv_csr_noalloc(10, 10, 134_217_729, 1, 1, 1, 1, 1, None)
    assert st == _abi.E_TOO_LARGE
    assert "134,217,728" in L.pava_last_error().decode()
    assert L.pava_spmv_csr_noalloc(-1, 10, 0, 1, 1, 1, 1, 1, None) == _abi.E_INVALID_ARG


def test_destroy_null_handles_are_no_ops():
    L = _abi.gpu()
    assert L.pava_destroy(None) == 0
    assert L.pava_batch_destroy(None) == 0


def test_generators_reject_bad_sizes():
    H = _abi.host()
    rp = np.zeros(8, np.int32)
    assert H.pava_gen_powerlaw_rowptr(-1, 5, 16.0, 1.5, 100, 0.02, 1, rp.ctypes.data) < 0
    assert H.pava_gen_banded_rowptr(-3, 4, 2, rp.ctypes.data) < 0
    assert M.laplace2d(4).nnz == 5 * 16 - 4 * 4
