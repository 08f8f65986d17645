"""Python mirror of the reference's engine interface, backed by the CUDA engine.

* ``SpMatrix``             -- a converted matrix on the GPU (pava_create / pava_spmv, and
  pava_spmm for k right-hand sides on the CSR row-group form)
* ``Batch``                -- many independent matrices as one block-diagonal union, one
  launch per SpMV, replayable from a CUDA graph (pava_batch_*)
* ``autotune``             -- exhaustive search over the candidate forms (pava_autotune)
* ``AnonymousLibHandle``   -- the CSR5 handle of csr5/anonymouslib_avx512.h:14-276 (inputCSR,
  setX, setSigma, asCSR5, spmv, asCSR, destroy), same names, argument meaning and status codes
* ``conduct_cvr`` / ``conduct_csr5`` -- the engine entry points of cvr/cvr.h:1953 and
  csr5/csr5.h:72, same arguments; they print the reference's ``Performance`` line
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from .matrices import CSR

FORMATS = {"csr": _abi.FORMAT_CSR, "csr5": _abi.FORMAT_CSR5, "cvr": _abi.FORMAT_CVR,
           "sell": _abi.FORMAT_SELL}


def _torch():
    import torch
    return torch


def _stream_ptr(stream) -> int | None:
    if stream is None:
        torch = _torch()
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


class SpMatrix:
    """A CSR matrix converted on the GPU into ``format`` ('cvr', 'csr5', 'sell' or 'csr').

    ``spmv(x)`` takes a CUDA tensor (float64 for FP64 handles) and returns y (float64).
    ``spmv_host(x)`` is the end-to-end form on host arrays.
    """

    def __init__(self, A: CSR, format: str = "cvr", steps: int = 0, sigma: int = 0,
                 tiles_per_chunk: int = 0, precision: int = _abi.PREC_FP64,
                 index_mode: int = _abi.INDEX_I32, lanes_per_row: int = 0,
                 col_lanes: int = 0, cols_per_lane: int = 0, rows_per_tile: int = 0,
                 x_window: int = 0, stream=None, device_arrays=None):
        L = _abi.gpu()
        self.m, self.n, self.nnz = A.m, A.n, A.nnz
        self.format = format
        self.precision = precision
        csr = _abi.PavaCsr()
        csr.m, csr.n, csr.nnz = A.m, A.n, A.nnz
        if device_arrays is not None:  # (rp, ci, v) CUDA tensors
            rp, ci, v = device_arrays
            csr.row_ptr, csr.col_idx, csr.vals = rp.data_ptr(), ci.data_ptr(), v.data_ptr()
            csr.on_device = 1
        else:
            self._keep = (np.ascontiguousarray(A.rp, np.int32), np.ascontiguousarray(A.ci, np.int32),
                          np.ascontiguousarray(A.v, np.float64))
            csr.row_ptr = self._keep[0].ctypes.data
            csr.col_idx = self._keep[1].ctypes.data
            csr.vals = self._keep[2].ctypes.data
            csr.on_device = 0
        opts = _abi.PavaOpts(steps, sigma, tiles_per_chunk, precision, index_mode, lanes_per_row,
                             col_lanes, cols_per_lane, rows_per_tile, x_window)
        h = _abi.c_void_p()
        _abi.check(L.pava_create(ctypes.byref(csr), FORMATS[format], ctypes.byref(opts),
                                 _abi.c_void_p(_stream_ptr(stream) if stream is not None else None),
                                 ctypes.byref(h)))
        self._h = h
        self._keep = None

    # -- info ---------------------------------------------------------------------------
    def info(self) -> dict:
        inf = _abi.PavaInfo()
        _abi.check(_abi.gpu().pava_get_info(self._h, ctypes.byref(inf)))
        return {f: getattr(inf, f) for f, _ in _abi.PavaInfo._fields_}

    # -- SpMV ---------------------------------------------------------------------------
    def spmv(self, x, y=None, stream=None):
        torch = _torch()
        if y is None:
            y = torch.empty(self.m, dtype=torch.float64, device=x.device)
        want = torch.float32 if self.precision == _abi.PREC_FP32C else torch.float64
        if x.dtype != want or not x.is_cuda or not x.is_contiguous():
            raise TypeError(f"x must be a contiguous CUDA {want} tensor")
        if y.dtype != torch.float64 or not y.is_cuda or y.numel() < self.m:
            raise TypeError("y must be a CUDA float64 tensor of m entries")
        _abi.check(_abi.gpu().pava_spmv(self._h, x.data_ptr(), y.data_ptr(),
                                        _abi.c_void_p(_stream_ptr(stream))))
        return y

    def spmm(self, X, Y=None, stream=None):
        """Y = A X for a row-major (n, k) CUDA tensor X (CSR handles, k <= 128; SELL handles,
        k <= 64); Y is (m, k) float64."""
        torch = _torch()
        want = torch.float32 if self.precision == _abi.PREC_FP32C else torch.float64
        if X.dim() != 2 or X.dtype != want or not X.is_cuda or X.stride(1) != 1:
            raise TypeError(f"X must be a row-major 2-D CUDA {want} tensor")
        k = X.shape[1]
        if Y is None:
            Y = torch.empty((self.m, k), dtype=torch.float64, device=X.device)
        if Y.dtype != torch.float64 or Y.dim() != 2 or Y.stride(1) != 1:
            raise TypeError("Y must be a row-major 2-D CUDA float64 tensor")
        _abi.check(_abi.gpu().pava_spmm(self._h, k, X.data_ptr(), X.stride(0), Y.data_ptr(),
                                        Y.stride(0), _abi.c_void_p(_stream_ptr(stream))))
        return Y

    def spmv_raw(self, x_ptr: int, y_ptr: int, stream_ptr: int | None, stage: int = 0) -> None:
        """pava_spmv_stage on raw device pointers: stage 1 = SpMV kernel, 2 = carry fixup,
        0 = both."""
        _abi.check(_abi.gpu().pava_spmv_stage(self._h, x_ptr, y_ptr, _abi.c_void_p(stream_ptr),
                                              stage))

    def spmv_host(self, x, y=None, stream=None):
        """End-to-end: host x -> device -> SpMV -> host y (numpy arrays or pinned tensors)."""
        xa = x
        if isinstance(x, np.ndarray):
            want = np.float32 if self.precision == _abi.PREC_FP32C else np.float64
            xa = np.ascontiguousarray(x, want)
            xp = xa.ctypes.data
        else:
            xp = x.data_ptr()
        if y is None:
            y = np.empty(self.m, np.float64)
        yp = y.ctypes.data if isinstance(y, np.ndarray) else y.data_ptr()
        sp = _stream_ptr(stream) if stream is not None else None
        _abi.check(_abi.gpu().pava_spmv_host(self._h, xp, yp, _abi.c_void_p(sp)))
        return y

    def spmv_host_async(self, x, y, stream=None):
        """Pipelined end-to-end SpMV on pinned host tensors (pava_spmv_host_async): returns at
        once; consecutive calls overlap their copies and SpMVs.  x and y must stay untouched
        until wait() (or until `stream` reaches the call)."""
        sp = _stream_ptr(stream) if stream is not None else None
        _abi.check(_abi.gpu().pava_spmv_host_async(self._h, x.data_ptr(), y.data_ptr(),
                                                   _abi.c_void_p(sp)))
        return y

    def wait(self):
        _abi.check(_abi.gpu().pava_spmv_host_wait(self._h))

    def close(self):
        if getattr(self, "_h", None):
            _abi.gpu().pava_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- autotuner and batches ------------------------------------------------------------------

FORMAT_NAMES = {v: k for k, v in FORMATS.items()}
OPT_KEYS = [f for f, _ in _abi.PavaOpts._fields_]


def _csr_struct(A: CSR, keep: list):
    csr = _abi.PavaCsr()
    csr.m, csr.n, csr.nnz = A.m, A.n, A.nnz
    arrs = (np.ascontiguousarray(A.rp, np.int32), np.ascontiguousarray(A.ci, np.int32),
            np.ascontiguousarray(A.v, np.float64))
    keep.append(arrs)
    csr.row_ptr, csr.col_idx, csr.vals = (a.ctypes.data for a in arrs)
    csr.on_device = 0
    return csr


def _opts_dict(o) -> dict:
    return {k: getattr(o, k) for k in OPT_KEYS}


def autotune(A: CSR, k: int = 1, precision: int = _abi.PREC_FP64, reps: int = 5):
    """Exhaustive search (pava_autotune): returns (entries, best_index); each entry is a dict
    with the form's name, its options, the median ms (< 0 if it failed) and the status."""
    keep = []
    csr = _csr_struct(A, keep)
    cap = 128
    ents = (_abi.PavaTuneEntry * cap)()
    n, best = _abi.c_int(), _abi.c_int()
    _abi.check(_abi.gpu().pava_autotune(ctypes.byref(csr), k, precision, reps, ents, cap,
                                        ctypes.byref(n), ctypes.byref(best)))
    out = [{"format": FORMAT_NAMES[e.format], "opts": _opts_dict(e.opts), "ms": e.ms,
            "status": e.status} for e in ents[: n.value]]
    return out, best.value


class Batch:
    """Many independent CSR matrices as one block-diagonal union on the GPU.

    ``format`` is 'cvr', 'csr5', 'csr' or 'auto' (autotuned over the candidate forms).  x and
    y of the batch are the matrices' vectors concatenated; ``layout()`` gives the offsets.
    ``k`` > 1 tunes the batch for k right-hand sides per matrix (``spmm``: X and Y are the
    matrices' n_i x k and m_i x k blocks stacked, row-major); that takes the 'csr' or 'auto'
    form.
    """

    def __init__(self, mats, format: str = "auto", precision: int = _abi.PREC_FP64, k: int = 1,
                 **opts):
        keep = []
        arr = (_abi.PavaCsr * len(mats))()
        for i, A in enumerate(mats):
            arr[i] = _csr_struct(A, keep)
        o = _abi.PavaOpts()
        o.precision = precision
        for key, val in opts.items():
            setattr(o, key, val)
        fmt = -1 if format == "auto" else FORMATS[format]
        h = _abi.c_void_p()
        _abi.check(_abi.gpu().pava_batch_create_spmm(len(mats), arr, k, fmt, ctypes.byref(o),
                                                     None, ctypes.byref(h)))
        self._h = h
        self.k = k
        self.count = len(mats)
        self.precision = precision
        xo = np.zeros(self.count + 1, np.int64)
        yo = np.zeros(self.count + 1, np.int64)
        zo = np.zeros(self.count + 1, np.int64)
        _abi.check(_abi.gpu().pava_batch_layout(h, xo.ctypes.data, yo.ctypes.data, zo.ctypes.data))
        self.x_offsets, self.y_offsets, self.nnz_offsets = xo, yo, zo
        self.n, self.m, self.nnz = int(xo[-1]), int(yo[-1]), int(zo[-1])

    def chosen(self):
        f = _abi.c_int()
        o = _abi.PavaOpts()
        _abi.check(_abi.gpu().pava_batch_get(self._h, ctypes.byref(f), ctypes.byref(o), None))
        return FORMAT_NAMES[f.value], _opts_dict(o)

    def info(self) -> dict:
        inf = _abi.PavaInfo()
        _abi.check(_abi.gpu().pava_batch_get(self._h, None, None, ctypes.byref(inf)))
        return {f: getattr(inf, f) for f, _ in _abi.PavaInfo._fields_}

    def _check_xy(self, x, y):
        torch = _torch()
        want = torch.float32 if self.precision == _abi.PREC_FP32C else torch.float64
        if x.dtype != want or not x.is_cuda or x.numel() < self.n:
            raise TypeError(f"x must be a CUDA {want} tensor of {self.n} entries")
        if y.dtype != torch.float64 or not y.is_cuda or y.numel() < self.m:
            raise TypeError(f"y must be a CUDA float64 tensor of {self.m} entries")

    def spmv(self, x, y=None, stream=None):
        torch = _torch()
        if y is None:
            y = torch.empty(self.m, dtype=torch.float64, device=x.device)
        self._check_xy(x, y)
        _abi.check(_abi.gpu().pava_batch_spmv(self._h, x.data_ptr(), y.data_ptr(),
                                              _abi.c_void_p(_stream_ptr(stream))))
        return y

    def capture(self, x, y):
        """Records the SpMV on (x, y) into the batch's CUDA graph."""
        self._check_xy(x, y)
        self._graph_xy = (x, y)
        _abi.check(_abi.gpu().pava_batch_capture(self._h, x.data_ptr(), y.data_ptr()))

    def _check_XY(self, X, Y):
        torch = _torch()
        want = torch.float32 if self.precision == _abi.PREC_FP32C else torch.float64
        if X.dim() != 2 or X.dtype != want or not X.is_cuda or X.shape[0] < self.n or X.stride(1) != 1:
            raise TypeError(f"X must be a CUDA {want} matrix of {self.n} row-major rows")
        if (Y.dim() != 2 or Y.dtype != torch.float64 or not Y.is_cuda or Y.shape[0] < self.m
                or Y.stride(1) != 1 or Y.shape[1] != X.shape[1]):
            raise TypeError(f"Y must be a CUDA float64 matrix of {self.m} row-major rows and "
                            "X's columns")

    def spmm(self, X, Y=None, stream=None):
        """Y = U X for the whole batch: X stacks the matrices' n_i x k right-hand sides."""
        torch = _torch()
        if Y is None:
            Y = torch.empty((self.m, X.shape[1]), dtype=torch.float64, device=X.device)
        self._check_XY(X, Y)
        _abi.check(_abi.gpu().pava_batch_spmm(self._h, X.shape[1], X.data_ptr(), X.stride(0),
                                              Y.data_ptr(), Y.stride(0),
                                              _abi.c_void_p(_stream_ptr(stream))))
        return Y

    def capture_spmm(self, X, Y):
        """Records the SpMM on (X, Y) into the batch's CUDA graph."""
        self._check_XY(X, Y)
        self._graph_xy = (X, Y)
        _abi.check(_abi.gpu().pava_batch_capture_spmm(self._h, X.shape[1], X.data_ptr(),
                                                      X.stride(0), Y.data_ptr(), Y.stride(0)))

    def replay(self, stream=None):
        _abi.check(_abi.gpu().pava_batch_replay(self._h, _abi.c_void_p(_stream_ptr(stream))))

    def split(self, y):
        """The per-matrix slices of a batch vector y."""
        return [y[self.y_offsets[i]: self.y_offsets[i + 1]] for i in range(self.count)]

    def close(self):
        if getattr(self, "_h", None):
            _abi.gpu().pava_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- the reference's CSR5 handle ----------------------------------------------------------

ANONYMOUSLIB_SUCCESS = 0
ANONYMOUSLIB_UNKOWN_FORMAT = -1
ANONYMOUSLIB_UNSUPPORTED_CSR5_OMEGA = -2
ANONYMOUSLIB_CSR_TO_CSR5_FAILED = -3
ANONYMOUSLIB_UNSUPPORTED_CSR_SPMV = -4
ANONYMOUSLIB_UNSUPPORTED_VALUE_TYPE = -5
ANONYMOUSLIB_FORMAT_CSR = 0
ANONYMOUSLIB_FORMAT_CSR5 = 1


class AnonymousLibHandle:
    """anonymouslibHandle<int, unsigned, double> (csr5/anonymouslib_avx512.h:14-276) on the
    GPU.  Unlike the reference, asCSR5 leaves the caller's arrays untouched and spmv writes
    every row of y (no accumulation across calls)."""

    def __init__(self, m: int, n: int):
        self._m, self._n = int(m), int(n)
        self._format = ANONYMOUSLIB_FORMAT_CSR
        self._csr = None
        self._x = None
        self._sigma = 16
        self._mat = None

    def warmup(self) -> int:
        return ANONYMOUSLIB_SUCCESS

    def inputCSR(self, nnz, csr_row_pointer, csr_column_index, csr_value) -> int:
        self._csr = CSR(self._m, self._n, np.ascontiguousarray(csr_row_pointer, np.int32),
                        np.ascontiguousarray(csr_column_index, np.int32)[:nnz],
                        np.ascontiguousarray(csr_value, np.float64)[:nnz])
        self._format = ANONYMOUSLIB_FORMAT_CSR
        return ANONYMOUSLIB_SUCCESS

    def setX(self, x) -> int:
        self._x = np.ascontiguousarray(x, np.float64)
        return ANONYMOUSLIB_SUCCESS

    def setSigma(self, sigma: int) -> None:
        self._sigma = int(sigma)

    def asCSR5(self) -> int:
        if self._format == ANONYMOUSLIB_FORMAT_CSR5:
            return ANONYMOUSLIB_SUCCESS
        try:
            self._mat = SpMatrix(self._csr, "csr5", sigma=self._sigma)
        except _abi.PavaError as e:
            if e.status == _abi.E_UNSUPPORTED_PARAMS:
                return ANONYMOUSLIB_UNSUPPORTED_CSR5_OMEGA
            return ANONYMOUSLIB_CSR_TO_CSR5_FAILED
        self._format = ANONYMOUSLIB_FORMAT_CSR5
        return ANONYMOUSLIB_SUCCESS

    def spmv(self, alpha: float, y) -> int:
        if self._format == ANONYMOUSLIB_FORMAT_CSR:
            return ANONYMOUSLIB_UNSUPPORTED_CSR_SPMV
        out = self._mat.spmv_host(self._x)
        y[: self._m] = out  # alpha is not applied, as in csr5_spmv_avx512.h:334
        return ANONYMOUSLIB_SUCCESS

    def asCSR(self) -> int:
        if self._mat is not None:
            self._mat.close()
            self._mat = None
        self._format = ANONYMOUSLIB_FORMAT_CSR
        return ANONYMOUSLIB_SUCCESS

    def destroy(self) -> int:
        return self.asCSR()


# ---- engine entry points ------------------------------------------------------------------

def _ptr(a):
    return a.ctypes.data


def conduct_cvr(numRows, numCols, nItems_raw, h_rowDelimiters, h_cols, h_val, h_vec, refOut,
                alpha, matrixName, numIterations) -> int:
    """conduct_cvr (cvr/cvr.h:1953): convert, one checked SpMV into refOut, numIterations
    timed SpMVs, print the Performance line.  Arrays are numpy; refOut is written in place."""
    rp = np.ascontiguousarray(h_rowDelimiters, np.int32)
    ci = np.ascontiguousarray(h_cols, np.int32)
    v = np.ascontiguousarray(h_val, np.float64)
    x = np.ascontiguousarray(h_vec, np.float64)
    assert refOut.dtype == np.float64 and refOut.flags.c_contiguous
    return _abi.gpu().conduct_cvr_gpu(numRows, numCols, nItems_raw, _ptr(rp), _ptr(ci), _ptr(v),
                                      _ptr(x), _ptr(refOut), int(alpha),
                                      str(matrixName).encode(), numIterations)


def conduct_csr5(m, n, nnzA, csrRowPtrA, csrColIdxA, csrValA, x, y, alpha, matrixName,
                 numIterations) -> int:
    """conduct_csr5 (csr5/csr5.h:72): same contract as conduct_cvr, CSR5 format."""
    rp = np.ascontiguousarray(csrRowPtrA, np.int32)
    ci = np.ascontiguousarray(csrColIdxA, np.int32)
    v = np.ascontiguousarray(csrValA, np.float64)
    xx = np.ascontiguousarray(x, np.float64)
    assert y.dtype == np.float64 and y.flags.c_contiguous
    return _abi.gpu().conduct_csr5_gpu(m, n, nnzA, _ptr(rp), _ptr(ci), _ptr(v), _ptr(xx),
                                       _ptr(y), float(alpha), str(matrixName).encode(),
                                       numIterations)
