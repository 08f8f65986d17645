"""COO -> CSR on the device against the host conversion (pava_coo_to_csr): 0- and 1-based
input, shuffled entries with duplicates, symmetric expansion, empty rows, bad indices."""
import numpy as np
import pytest

from pava_b200 import _abi
from pava_b200 import matrices as M

pytestmark = pytest.mark.gpu


def _host_csr(m, n, r, c, v):
    rp = np.zeros(m + 1, np.int32)
    ci = np.empty(len(r), np.int32)
    vv = np.empty(len(r), np.float64)
    p = lambda a: a.ctypes.data_as(_abi.c_void_p)
    r = np.ascontiguousarray(r, np.int32)
    c = np.ascontiguousarray(c, np.int32)
    v = np.ascontiguousarray(v, np.float64)
    assert _abi.host().pava_coo_to_csr(m, n, len(r), p(r), p(c), p(v), p(rp), p(ci), p(vv)) == 0
    return rp, ci, vv


def _random_coo(m, n, nnz, seed):
    rng = np.random.default_rng(seed)
    r = rng.integers(0, m, nnz).astype(np.int32)
    c = rng.integers(0, n, nnz).astype(np.int32)
    r[: nnz // 10] = 3                      # a long row, and duplicates of (3, c)
    c[: nnz // 20] = 7
    v = rng.normal(size=nnz)
    return r, c, v


@pytest.mark.parametrize("base", [0, 1])
@pytest.mark.parametrize("m,n,nnz", [(1000, 1300, 20_000), (200_000, 200_000, 1_500_000), (5, 5, 0)])
def test_general(cuda, base, m, n, nnz):
    torch = cuda
    r, c, v = _random_coo(m, n, nnz, seed=m + base)
    rp, ci, vv = M.coo_to_csr_device(m, n, torch.from_numpy(r + base).cuda(),
                                     torch.from_numpy(c + base).cuda(), torch.from_numpy(v).cuda(),
                                     index_base=base)
    hrp, hci, hv = _host_csr(m, n, r, c, v)
    assert np.array_equal(rp.cpu().numpy(), hrp)
    assert np.array_equal(ci.cpu().numpy(), hci)
    assert np.array_equal(vv.cpu().numpy(), hv)


def test_symmetric_expansion(cuda):
    torch = cuda
    m = 50_000
    rng = np.random.default_rng(3)
    r = rng.integers(0, m, 300_000).astype(np.int32)
    c = rng.integers(0, m, 300_000).astype(np.int32)
    lo = np.minimum(r, c)
    hi = np.maximum(r, c)
    r, c = hi, lo                          # one triangle, diagonal included
    v = rng.normal(size=len(r))
    rp, ci, vv = M.coo_to_csr_device(m, m, torch.from_numpy(r + 1).cuda(),
                                     torch.from_numpy(c + 1).cuda(), torch.from_numpy(v).cuda(),
                                     index_base=1, symmetric=True)
    off = r != c
    er = np.concatenate([r, c[off]])
    ec = np.concatenate([c, r[off]])
    ev = np.concatenate([v, v[off]])
    hrp, hci, hv = _host_csr(m, m, er, ec, ev)
    assert np.array_equal(rp.cpu().numpy(), hrp)
    assert np.array_equal(ci.cpu().numpy(), hci)
    assert np.array_equal(vv.cpu().numpy(), hv)


def test_rejects_out_of_range(cuda):
    torch = cuda
    r = torch.tensor([0, 1, 2], dtype=torch.int32, device="cuda")
    c = torch.tensor([0, 5, 1], dtype=torch.int32, device="cuda")
    v = torch.ones(3, dtype=torch.float64, device="cuda")
    with pytest.raises(_abi.PavaError) as e:
        M.coo_to_csr_device(3, 5, r, c, v)      # column 5 == n
    assert e.value.status == _abi.E_INVALID_CSR
    with pytest.raises(_abi.PavaError) as e:
        M.coo_to_csr_device(3, 6, r, c, v, index_base=1)   # row 0 in a 1-based file
    assert e.value.status == _abi.E_INVALID_CSR
