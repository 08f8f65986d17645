"""The C ABI: the libraries load without a GPU and export every function include/*.h declares;
the host-side generators, Matrix Market I/O and COO->CSR behave.  No GPU compute here."""
import ctypes
import os
import re

import numpy as np
import pytest

from pava_b200 import _abi
from pava_b200 import matrices as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", text)
    skip = {"if", "for", "while", "sizeof", "return"}
    return sorted({n for n in names if n not in skip and (n.startswith("pava_") or n.startswith("conduct_"))})


def _exported(path):
    lib = ctypes.CDLL(path)
    return lib


@pytest.mark.parametrize("header,path", [("pava_gpu.h", _abi.gpu_lib_path()),
                                         ("pava_host.h", _abi.host_lib_path()),
                                         ("pava_probe.h", _abi.probe_lib_path())])
def test_library_exports_every_declared_symbol(header, path):
    names = _declared(header)
    assert len(names) >= (2 if header == "pava_probe.h" else 8)
    lib = _exported(path)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_the_headers():
    bound = ({n for n, _, _ in _abi.GPU_SYMBOLS} | {n for n, _, _ in _abi.HOST_SYMBOLS}
             | {n for n, _, _ in _abi.PROBE_SYMBOLS})
    declared = (set(_declared("pava_gpu.h")) | set(_declared("pava_host.h"))
                | set(_declared("pava_probe.h")))
    assert declared <= bound, sorted(declared - bound)


def test_status_strings_without_gpu():
    L = _abi.gpu()
    assert L.pava_status_string(_abi.E_INVALID_CSR) == b"invalid CSR"
    assert L.pava_status_string(0) == b"success"


def test_laplace2d_shape():
    A = M.laplace2d(512)
    assert A.m == 262144 and A.nnz == 1308672
    r = 512 * 100 + 7
    cols = A.ci[A.rp[r]:A.rp[r + 1]]
    assert list(cols) == [r - 512, r - 1, r, r + 1, r + 512]
    assert list(A.v[A.rp[r]:A.rp[r + 1]]) == [-1, -1, 4, -1, -1]


def test_generators_deterministic_and_sorted():
    a = M.powerlaw(20000, seed=5, cap=3000)
    b = M.powerlaw(20000, seed=5, cap=3000)
    assert np.array_equal(a.rp, b.rp) and np.array_equal(a.ci, b.ci) and np.array_equal(a.v, b.v)
    lens = np.diff(a.rp)
    assert 0.01 < np.mean(lens == 0) < 0.03
    for r in np.nonzero(lens > 1)[0][:500]:
        seg = a.ci[a.rp[r]:a.rp[r + 1]]
        assert np.all(np.diff(seg) > 0)
    assert a.ci.min() >= 0 and a.ci.max() < a.n


def test_stencil27_fp32_representable():
    A = M.stencil27(12)
    assert A.nnz == (3 * 12 - 2) ** 3
    assert np.array_equal(A.v.astype(np.float32).astype(np.float64), A.v)
    diag = np.array([A.v[A.rp[r] + np.searchsorted(A.ci[A.rp[r]:A.rp[r + 1]], r)] for r in range(A.m)])
    assert np.all(diag > 0)


def test_banded_random_blockdiag():
    B = M.banded(5000, 64, 24)
    assert np.all(np.diff(B.rp) == 24)
    r = np.repeat(np.arange(B.m), 24)
    assert np.all(np.abs(B.ci - r) <= 64)
    R = M.random_csr(3000, 4000, 12.0)
    assert abs(np.diff(R.rp).mean() - 12.0) < 0.5
    D = M.blockdiag(1000, 8, 64)
    assert D.ci.max() < 1000


def test_mtx_roundtrip_and_coo_to_csr(tmp_path):
    A = M.powerlaw(3000, seed=9, cap=500)
    p = str(tmp_path / "a.mtx")
    M.write_mtx(p, A)
    B = M.read_mtx(p)
    assert B.m == A.m and B.n == A.n
    assert np.array_equal(A.rp, B.rp) and np.array_equal(A.ci, B.ci)
    assert np.array_equal(A.v, B.v)


def test_mtx_symmetric_pattern_expansion(tmp_path):
    p = tmp_path / "s.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n% c\n3 3 3\n1 1\n2 1\n3 2\n")
    B = M.read_mtx(str(p))
    assert list(B.rp) == [0, 2, 4, 5]
    assert list(B.ci) == [0, 1, 0, 2, 1]
    assert np.all(B.v == 1.0)


def test_init_vectors():
    x, y, yr = M.init_vectors(4, 5)
    assert list(x) == [0, 1, 2, 0, 1] and not y.any() and not yr.any()
