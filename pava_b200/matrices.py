"""Seeded synthetic matrices of the benchmark configurations, and Matrix Market I/O.

Thin numpy wrappers over the host library (include/pava_host.h).  The workloads:

* ``laplace2d(512)``          -- 2-D 5-point Laplacian, 262,144 rows, 1,308,672 nnz
* ``powerlaw(4194304, ...)``  -- lognormal row lengths (mean 16, sigma 1.5, cap 200,000, 2 %
  empty rows), uniform distinct columns, N(0,1) values: ~64 M nnz
* ``stencil27(128)``          -- 3-D 27-point stencil, 2,097,152 rows, 55,742,968 nnz, values
  exactly representable in FP32
* ``banded(1048576, 64, 24)`` -- 24 distinct columns in a half-bandwidth-64 band
* ``random_csr`` / ``blockdiag`` -- the batched and selector families

The reference benchmarks on SuiteSparse/SNAP files; these seeded generators stand in for
them with the shapes, sizes and value distributions the configurations state.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _abi


@dataclass
class CSR:
    m: int
    n: int
    rp: np.ndarray   # int32, m + 1
    ci: np.ndarray   # int32, nnz
    v: np.ndarray    # float64, nnz

    @property
    def nnz(self) -> int:
        return int(self.rp[-1])


def _p(a):
    return a.ctypes.data_as(_abi.c_void_p)


def _rc(rc):
    if rc != 0:
        raise RuntimeError(f"pava host library returned {rc}")


def _alloc(m):
    return np.zeros(m + 1, np.int32)


def _fill(rp):
    nnz = int(rp[-1])
    return np.empty(nnz, np.int32), np.empty(nnz, np.float64)


def laplace2d(grid: int) -> CSR:
    H = _abi.host()
    m = grid * grid
    rp = _alloc(m)
    _rc(H.pava_gen_laplace2d_rowptr(grid, _p(rp)))
    ci, v = _fill(rp)
    _rc(H.pava_gen_laplace2d_fill(grid, _p(rp), _p(ci), _p(v)))
    return CSR(m, m, rp, ci, v)


def powerlaw(m: int, n: int | None = None, mean: float = 16.0, sigma: float = 1.5,
             cap: int = 200_000, p_empty: float = 0.02, seed: int = 1) -> CSR:
    H = _abi.host()
    n = m if n is None else n
    rp = _alloc(m)
    _rc(H.pava_gen_powerlaw_rowptr(m, n, mean, sigma, cap, p_empty, seed, _p(rp)))
    ci, v = _fill(rp)
    _rc(H.pava_gen_powerlaw_fill(m, n, seed, _p(rp), _p(ci), _p(v)))
    return CSR(m, n, rp, ci, v)


def stencil27(grid: int, seed: int = 2) -> CSR:
    H = _abi.host()
    m = grid ** 3
    rp = _alloc(m)
    _rc(H.pava_gen_stencil27_rowptr(grid, _p(rp)))
    ci, v = _fill(rp)
    _rc(H.pava_gen_stencil27_fill(grid, seed, _p(rp), _p(ci), _p(v)))
    return CSR(m, m, rp, ci, v)


def banded(m: int, halfbw: int = 64, per_row: int = 24, seed: int = 3) -> CSR:
    H = _abi.host()
    rp = _alloc(m)
    _rc(H.pava_gen_banded_rowptr(m, halfbw, per_row, _p(rp)))
    ci, v = _fill(rp)
    _rc(H.pava_gen_banded_fill(m, halfbw, seed, _p(rp), _p(ci), _p(v)))
    return CSR(m, m, rp, ci, v)


def random_csr(m: int, n: int | None = None, mean: float = 12.0, seed: int = 4) -> CSR:
    H = _abi.host()
    n = m if n is None else n
    rp = _alloc(m)
    _rc(H.pava_gen_random_rowptr(m, n, mean, seed, _p(rp)))
    ci, v = _fill(rp)
    _rc(H.pava_gen_random_fill(m, n, seed, _p(rp), _p(ci), _p(v)))
    return CSR(m, n, rp, ci, v)


def blockdiag(m: int, bmin: int = 8, bmax: int = 64, seed: int = 5) -> CSR:
    H = _abi.host()
    rp = _alloc(m)
    _rc(H.pava_gen_blockdiag_rowptr(m, bmin, bmax, seed, _p(rp)))
    ci, v = _fill(rp)
    _rc(H.pava_gen_blockdiag_fill(m, seed, _p(rp), _p(ci), _p(v)))
    return CSR(m, m, rp, ci, v)


def uniform(n: int, lo: float = -1.0, hi: float = 1.0, seed: int = 0,
            fp32: bool = False) -> np.ndarray:
    x = np.empty(n, np.float64)
    _rc(_abi.host().pava_gen_uniform(n, lo, hi, seed, int(fp32), _p(x)))
    return x


def init_vectors(m: int, n: int):
    """initVectors (utils/basicMatrix.cpp:499-520): x[i] = i % 3, y = y_ref = 0."""
    x = np.empty(n)
    y = np.empty(m)
    yr = np.empty(m)
    _abi.host().pava_init_vectors(m, n, _p(x), _p(y), _p(yr))
    return x, y, yr


def sell_padded_elements(A: CSR) -> int:
    """Elements the SELL form stores for A: per slice of 32 rows (the last one filled up with
    empty rows), 32 x its longest row rounded up to a multiple of 4."""
    lens = np.diff(np.asarray(A.rp, np.int64))
    ns = (A.m + 31) // 32
    lens = np.concatenate([lens, np.zeros(ns * 32 - A.m, np.int64)]).reshape(ns, 32)
    return int(((lens.max(axis=1) + 3) // 4).sum()) * 128 if ns else 0


def sell_accepts(A: CSR) -> bool:
    """Whether pava_create takes A in the SELL form: its padding at most doubles the stored
    elements (plus one block of 128 per slice), PAVA_E_UNSUPPORTED_PARAMS otherwise."""
    return sell_padded_elements(A) <= 2 * A.nnz + 128 * ((A.m + 31) // 32)


def from_arrays(m, n, rp, ci, v) -> CSR:
    return CSR(int(m), int(n), np.ascontiguousarray(rp, np.int32),
               np.ascontiguousarray(ci, np.int32), np.ascontiguousarray(v, np.float64))


def read_mtx(path: str) -> CSR:
    """Matrix Market -> sorted 0-based CSR (readCOOMatrix + convertCOO2CSR,
    utils/basicMatrix.cpp:63-415, with the 1-based indices converted explicitly)."""
    H = _abi.host()
    m, n, k, sym = _abi.c_int(), _abi.c_int(), _abi.c_int(), _abi.c_int()
    nz = _abi.c_ll()
    _rc(H.pava_mtx_info(path.encode(), m, n, nz, k, sym))
    rows = np.empty(nz.value, np.int32)
    cols = np.empty(nz.value, np.int32)
    vals = np.empty(nz.value, np.float64)
    got = _abi.c_ll()
    _rc(H.pava_mtx_read(path.encode(), _p(rows), _p(cols), _p(vals), got))
    rows, cols, vals = rows[:got.value], cols[:got.value], vals[:got.value]
    rp = np.empty(m.value + 1, np.int32)
    ci = np.empty(got.value, np.int32)
    v = np.empty(got.value, np.float64)
    _rc(H.pava_coo_to_csr(m.value, n.value, got.value, _p(rows), _p(cols), _p(vals), _p(rp),
                          _p(ci), _p(v)))
    return CSR(m.value, n.value, rp, ci, v)


def write_mtx(path: str, A: CSR) -> None:
    _rc(_abi.host().pava_mtx_write(path.encode(), A.m, A.n, _p(A.rp), _p(A.ci), _p(A.v)))


def coo_to_csr_device(m: int, n: int, rows, cols, vals, index_base: int = 0,
                      symmetric: bool = False):
    """COO on the GPU -> sorted CSR on the GPU (pava_coo_to_csr_device).  rows / cols are
    int32 CUDA tensors, vals a float64 CUDA tensor.  Returns (rp, ci, v) CUDA tensors."""
    import torch
    A = _abi.PavaCsr()
    _abi.check(_abi.gpu().pava_coo_to_csr_device(m, n, rows.numel(), rows.data_ptr(),
                                                 cols.data_ptr(), vals.data_ptr(), index_base,
                                                 int(symmetric), None, A))
    try:
        out = []
        for ptr, cnt, ts, dt in ((A.row_ptr, m + 1, "<i4", torch.int32),
                                 (A.col_idx, A.nnz, "<i4", torch.int32),
                                 (A.vals, A.nnz, "<f8", torch.float64)):
            t = torch.empty(cnt, dtype=dt, device="cuda")
            if cnt:
                t.copy_(torch.as_tensor(_DevView(ptr, cnt, ts), device="cuda"))
            out.append(t)
        return tuple(out)
    finally:
        _abi.gpu().pava_free_device_csr(A)


class _DevView:
    """A device buffer seen through the CUDA array interface (no copy)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3}
