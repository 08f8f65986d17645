"""The allocation-free entry point pava_spmv_csr_noalloc, through the C ABI.

It serves callers that may not call the CUDA allocator: a framework owns their device memory
and hands them only pre-allocated buffers, so they cannot create a handle (conversion
allocates).  The entry point reads their device CSR directly and keeps its scratch in a fixed
1 MiB array compiled into the library.  Here the test plays that caller: its inputs and outputs
are allocated beforehand (by torch), and the entry point is called twice in a row on each
matrix.  Both results must agree with the handle-based pava_spmv (CSR5 form) within the FP64
tolerance of the other parity tests, 1e-12 relative per row, and with the oracle's product.

This file is named to be collected last, so that a run stopping at the first failure has run
every other test first; it also passes on its own in a fresh process."""
import numpy as np
import pytest

from oracle import oracle as O
from pava_b200 import _abi
from pava_b200 import matrices as M
from pava_b200.api import SpMatrix

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _device_csr(torch, A):
    return (torch.from_numpy(A.rp).cuda(), torch.from_numpy(A.ci).cuda(),
            torch.from_numpy(A.v).cuda())


def _noalloc(torch, A, rp, ci, v, x, y):
    st = _abi.gpu().pava_spmv_csr_noalloc(A.m, A.n, A.nnz, rp.data_ptr(), ci.data_ptr(),
                                          v.data_ptr(), x.data_ptr(), y.data_ptr(),
                                          torch.cuda.current_stream().cuda_stream)
    assert st == 0, _abi.gpu().pava_status_string(st)
    torch.cuda.synchronize()
    return y.cpu().numpy().copy()


CASES = [
    ("powerlaw_long_rows", lambda: M.powerlaw(150_000, mean=16.0, sigma=2.0, cap=40_000, seed=61)),
    ("laplace2d_512", lambda: M.laplace2d(512)),
    ("mostly_empty", lambda: M.powerlaw(40_000, mean=6.0, p_empty=0.7, seed=62)),
    ("one_row", lambda: M.from_arrays(1, 9000, [0, 9000], np.arange(9000, dtype=np.int32),
                                      np.random.default_rng(63).normal(size=9000))),
    ("all_empty", lambda: M.from_arrays(50, 50, np.zeros(51, np.int32), [], [])),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_handle_path_twice(cuda, name, make):
    torch = cuda
    A = make()
    x_host = M.uniform(A.n, seed=64)
    rp, ci, v = _device_csr(torch, A)
    x = torch.from_numpy(x_host).cuda()
    y = torch.full((A.m,), float("nan"), dtype=torch.float64, device="cuda")
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x_host)
    # the existing entry point (handle, CSR5 form) on the same inputs
    ref = SpMatrix(A, "csr5").spmv(x).cpu().numpy()
    for _ in range(2):  # two calls in a row share (and reuse) the scratch array
        y.fill_(float("nan"))
        got = _noalloc(torch, A, rp, ci, v, x, y)
        assert O.rel_error(got, ref, ab, TOL)[0] == 0
        assert O.rel_error(got, yr, ab, TOL)[0] == 0


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    torch = cuda
    # 134,217,729 nonzeros need 32,769 chunks of 4,096: one more than the scratch holds; the
    # call returns before reading any array, so none are passed
    st = _abi.gpu().pava_spmv_csr_noalloc(10, 10, 134_217_729, 1, 1, 1, 1, 1,
                                          torch.cuda.current_stream().cuda_stream)
    assert st == _abi.E_TOO_LARGE
