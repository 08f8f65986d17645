"""ORACLE -- test infrastructure only.

ctypes bindings for the oracle libraries built by oracle/Makefile:

* ``liboracle.so``       -- the plain-C restatement of the reference's CVR and CSR5 engines
  (cvr/cvr.h; csr5/anonymouslib_avx512.h + csr5/detail/avx512/*.h), the long-double CSR
  reference and the error metric.  Portable.
* ``_ref/libpava_ref.so`` -- the reference engines themselves, compiled from the reference tree
  with an intrinsic shim.  Needs an AVX-512 CPU; ``have_ref()`` says whether it can be used.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this
module, and only as the oracle the GPU results are compared with or as the reported CPU
baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_dptr = ctypes.POINTER(ctypes.c_double)


def reference_tree() -> str:
    """The reference's source tree: PAVA_REF, else a `reference` directory beside this
    repository's own directory."""
    return os.environ.get("PAVA_REF") or os.path.join(os.path.dirname(os.path.dirname(HERE)),
                                                      "reference")


def build(ref: bool = True) -> None:
    """Builds liboracle.so, and _ref/libpava_ref.so when the reference tree is present."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    ref_tree = reference_tree()
    if ref and os.path.isfile(os.path.join(ref_tree, "cvr", "cvr.h")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"PAVA_REF={ref_tree}"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        L = ctypes.CDLL(path)
        L.oracle_csr_ref.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p]
        L.oracle_csr_ref.restype = None
        L.oracle_rel_error.argtypes = [ctypes.c_int, _f64p, _f64p, _f64p, ctypes.c_double,
                                       _dptr, _dptr]
        L.oracle_rel_error.restype = ctypes.c_longlong
        L.oracle_check_results.argtypes = [ctypes.c_int, _f64p, _f64p]
        L.oracle_check_results.restype = ctypes.c_longlong
        L.oracle_cvr_run.argtypes = [ctypes.c_int] * 4 + [_i32p, _i32p, _f64p, _f64p, _f64p,
                                                          _dptr, _dptr, ctypes.c_int]
        L.oracle_cvr_run.restype = ctypes.c_int
        L.oracle_csr5_run.argtypes = [ctypes.c_int] * 5 + [_i32p, _i32p, _f64p, _f64p, _f64p,
                                                           _dptr, _dptr, ctypes.c_int]
        L.oracle_csr5_run.restype = ctypes.c_int
        L.oracle_cvr_padded.argtypes = [ctypes.c_int]
        L.oracle_cvr_padded.restype = ctypes.c_int
        L.oracle_cvr_record_len.argtypes = [ctypes.c_int, ctypes.c_int]
        L.oracle_cvr_record_len.restype = ctypes.c_longlong
        L.oracle_cvr_convert.argtypes = [ctypes.c_int] * 3 + [_i32p, _i32p, _f64p, _f64p, _i32p,
                                                              _i32p, _i32p, _i32p, _i32p]
        L.oracle_cvr_convert.restype = None
        _LIB = L
    return _LIB


def have_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return "avx512f" in line.split()
    except OSError:
        pass
    return False


def have_ref() -> bool:
    return have_avx512() and os.path.exists(os.path.join(HERE, "_ref", "libpava_ref.so"))


def ref():
    """The reference engines compiled from the reference tree (AVX-512 hosts only)."""
    global _REF
    if _REF is None:
        if not have_ref():
            raise RuntimeError("oracle/_ref/libpava_ref.so unavailable (not built or no AVX-512)")
        L = ctypes.CDLL(os.path.join(HERE, "_ref", "libpava_ref.so"))
        L.pava_ref_cvr.argtypes = [ctypes.c_int] * 4 + [_i32p, _i32p, _f64p, _f64p, _f64p,
                                                        ctypes.c_int, _dptr, _dptr,
                                                        ctypes.c_void_p, ctypes.c_void_p,
                                                        ctypes.c_void_p, ctypes.c_longlong,
                                                        ctypes.c_void_p, ctypes.c_void_p,
                                                        ctypes.c_void_p]
        L.pava_ref_cvr.restype = ctypes.c_int
        L.pava_ref_cvr_record_len.argtypes = [ctypes.c_int, ctypes.c_int]
        L.pava_ref_cvr_record_len.restype = ctypes.c_longlong
        L.pava_ref_csr5.argtypes = [ctypes.c_int] * 5 + [_i32p, _i32p, _f64p, _f64p, _f64p,
                                                         ctypes.c_int, _dptr, _dptr] + \
            [ctypes.c_void_p] * 4 + [ctypes.c_int] + [ctypes.c_void_p] * 3
        L.pava_ref_csr5.restype = ctypes.c_int
        L.pava_ref_csr5_params.argtypes = [ctypes.c_int, ctypes.c_int, _i32p]
        L.pava_ref_csr5_params.restype = None
        _REF = L
    return _REF


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _csr_args(rp, ci, v):
    return (np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32),
            np.ascontiguousarray(v, np.float64))


def csr_ref(rp, ci, v, x):
    """Long-double CSR product (referenceSpMV, utils/basicMatrix.cpp:538, wider accumulator).
    Returns (y_ref, absum) where absum[i] = sum_j |a_ij x_j|."""
    rp, ci, v = _csr_args(rp, ci, v)
    m = len(rp) - 1
    y = np.zeros(m)
    a = np.zeros(m)
    lib().oracle_csr_ref(m, rp, ci, v, np.ascontiguousarray(x, np.float64), y, a)
    return y, a


def rel_error(y, y_ref, absum, tol=1e-12):
    """Cancellation-aware per-row relative error: |y-yref| / max(|yref|, sum|a_ij x_j|).
    Returns (rows over tol, max, mean)."""
    mx = ctypes.c_double()
    mean = ctypes.c_double()
    bad = lib().oracle_rel_error(len(y), np.ascontiguousarray(y, np.float64),
                                 np.ascontiguousarray(y_ref, np.float64),
                                 np.ascontiguousarray(absum, np.float64), tol,
                                 ctypes.byref(mx), ctypes.byref(mean))
    return int(bad), mx.value, mean.value


def check_results(y, y_ref):
    """checkResults (utils/basicMatrix.cpp:559-587): rows off by more than 1 %."""
    return int(lib().oracle_check_results(len(y), np.ascontiguousarray(y, np.float64),
                                          np.ascontiguousarray(y_ref, np.float64)))


def cvr_port(rp, ci, v, x, n=None, nthreads=8, iters=0):
    """Restated reference CVR: first SpMV after conversion.  Returns (y, convert_s, exec_s)."""
    rp, ci, v = _csr_args(rp, ci, v)
    m = len(rp) - 1
    n = len(x) if n is None else n
    y = np.zeros(m)
    cs, es = ctypes.c_double(), ctypes.c_double()
    rc = lib().oracle_cvr_run(nthreads, m, n, len(ci), rp, ci, v,
                              np.ascontiguousarray(x, np.float64), y, ctypes.byref(cs),
                              ctypes.byref(es), iters)
    if rc != 0:
        raise MemoryError("oracle_cvr_run failed")
    return y, cs.value, es.value


def csr5_port(rp, ci, v, x, n=None, nthreads=8, sigma=12, iters=0):
    """Restated reference CSR5 (omega 8): first SpMV after conversion."""
    rp, ci, v = _csr_args(rp, ci, v)
    m = len(rp) - 1
    n = len(x) if n is None else n
    y = np.zeros(m)
    cs, es = ctypes.c_double(), ctypes.c_double()
    rc = lib().oracle_csr5_run(nthreads, sigma, m, n, len(ci), rp, ci, v,
                               np.ascontiguousarray(x, np.float64), y, ctypes.byref(cs),
                               ctypes.byref(es), iters)
    if rc != 0:
        raise MemoryError("oracle_csr5_run failed")
    return y, cs.value, es.value


def cvr_port_layout(rp, ci, v, nthreads):
    """Restated CSR->CVR conversion; returns the layout arrays (vals, cols, rec, split,
    nnz_rows, final2) on the nnz padded to 16 into the last row, as the reference builds it."""
    rp, ci, v = _csr_args(rp, ci, v)
    m = len(rp) - 1
    nnz = len(ci)
    L = lib()
    nitems = L.oracle_cvr_padded(nnz)
    slack = 256
    rp2 = np.full(m + 1 + slack, nitems, np.int32)
    rp2[:m] = rp[:m]
    ci2 = np.zeros(nitems + slack, np.int32)
    ci2[:nnz] = ci
    v2 = np.zeros(nitems + slack)
    v2[:nnz] = v
    vals = np.zeros(nitems + slack)
    cols = np.zeros(nitems + slack, np.int32)
    rec = np.zeros(L.oracle_cvr_record_len(nthreads, m), np.int32)
    split = np.zeros(2 * nthreads + 16, np.int32)
    nnz_rows = np.zeros(4 * nthreads + 16, np.int32)
    final2 = np.zeros(16 * nthreads + 16, np.int32)
    L.oracle_cvr_convert(nthreads, m, nitems, rp2, ci2, v2, vals, cols, rec, split, nnz_rows,
                         final2)
    return (vals[:nitems], cols[:nitems], rec, split[:2 * nthreads], nnz_rows[:4 * nthreads],
            final2[:16 * nthreads])


def ref_cvr(rp, ci, v, x, n=None, nthreads=8, iters=0, layout=False):
    """The reference CVR (compiled from the reference tree): first SpMV after conversion.
    Returns (y, convert_s, exec_s[, layout tuple like cvr_port_layout])."""
    rp, ci, v = _csr_args(rp, ci, v)
    m = len(rp) - 1
    n = len(x) if n is None else n
    nnz = len(ci)
    R = ref()
    y = np.zeros(m)
    cs, es = ctypes.c_double(), ctypes.c_double()
    out = None
    if layout:
        nitems = (nnz if nnz % 16 == 0 else (nnz + 16) // 16 * 16)
        rl = R.pava_ref_cvr_record_len(nthreads, m)
        out = (np.zeros(nitems), np.zeros(nitems, np.int32), np.zeros(rl, np.int32),
               np.zeros(2 * nthreads, np.int32), np.zeros(4 * nthreads, np.int32),
               np.zeros(16 * nthreads, np.int32))
    rc = R.pava_ref_cvr(nthreads, m, n, nnz, rp, ci, v, np.ascontiguousarray(x, np.float64), y,
                        iters, ctypes.byref(cs), ctypes.byref(es),
                        _ptr(out[0]) if out else None, _ptr(out[1]) if out else None,
                        _ptr(out[2]) if out else None, len(out[2]) if out else 0,
                        _ptr(out[3]) if out else None, _ptr(out[4]) if out else None,
                        _ptr(out[5]) if out else None)
    if rc != 0:
        raise MemoryError("pava_ref_cvr failed")
    return (y, cs.value, es.value) + ((out,) if layout else ())


def ref_csr5(rp, ci, v, x, n=None, nthreads=8, sigma=12, iters=0, layout=False):
    """The reference CSR5 (compiled from the reference tree): first SpMV after asCSR5.
    Returns (y, convert_s, exec_s[, dict of tile arrays])."""
    rp, ci, v = _csr_args(rp, ci, v)
    m = len(rp) - 1
    n = len(x) if n is None else n
    nnz = len(ci)
    R = ref()
    y = np.zeros(m)
    cs, es = ctypes.c_double(), ctypes.c_double()
    par = np.zeros(4, np.int32)
    R.pava_ref_csr5_params(nnz, sigma, par)
    p, _, _, npk = (int(t) for t in par)
    d = None
    noff = ctypes.c_int(0)
    if layout:
        d = dict(tile_ptr=np.zeros(p + 1, np.uint32), tile_desc=np.zeros(p * 8 * npk, np.uint32),
                 desc_off_ptr=np.zeros(p + 1, np.int32), desc_off=np.zeros(nnz + 8, np.int32),
                 tcols=np.zeros(nnz, np.int32), tvals=np.zeros(nnz))
    rc = R.pava_ref_csr5(nthreads, sigma, m, n, nnz, rp, ci, v,
                         np.ascontiguousarray(x, np.float64), y, iters, ctypes.byref(cs),
                         ctypes.byref(es),
                         _ptr(d["tile_ptr"]) if d else None, _ptr(d["tile_desc"]) if d else None,
                         _ptr(d["desc_off_ptr"]) if d else None,
                         _ptr(d["desc_off"]) if d else None, nnz + 8 if d else 0,
                         ctypes.byref(noff), _ptr(d["tcols"]) if d else None,
                         _ptr(d["tvals"]) if d else None)
    if rc != 0:
        raise RuntimeError(f"pava_ref_csr5 failed with status {rc}")
    if d is not None:
        d["num_offsets"] = noff.value
        d["desc_off"] = d["desc_off"][:noff.value]
        return y, cs.value, es.value, d
    return y, cs.value, es.value
