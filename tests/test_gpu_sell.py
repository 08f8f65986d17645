"""The SELL form (32-row slices, one lane per row, streams staged through shared memory by
bulk copies) against the oracle on the shapes its conversion and its piece walk must get
right: slices longer than a shared-memory stage, runs of empty slices, ragged last slices,
more and fewer slices than resident warps, the padding threshold, and per-slice 16-bit bases.

Tolerances as in test_gpu_parity.py (FP64: 1e-12 relative per row, cancellation-aware) and
test_gpu_precision.py (FP32C: 1e-9)."""
import numpy as np
import pytest

from oracle import oracle as O
from pava_b200 import _abi
from pava_b200 import matrices as M
from pava_b200.api import SpMatrix

pytestmark = pytest.mark.gpu


def _run(torch, A, x, **kw):
    mat = SpMatrix(A, "sell", **kw)
    fp32 = kw.get("precision") == _abi.PREC_FP32C
    xd = torch.from_numpy(x).to("cuda", torch.float32 if fp32 else torch.float64)
    y = torch.full((A.m,), float("nan"), dtype=torch.float64, device="cuda")
    mat.spmv(xd, y)
    y1 = y.cpu().numpy().copy()
    mat.spmv(xd, y)
    assert np.array_equal(y1, y.cpu().numpy()), "repeated SpMV differs"
    info = mat.info()
    mat.close()
    return y1, info


def _check(y, A, x, tol):
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    bad, mx, _ = O.rel_error(y, yr, ab, tol)
    assert bad == 0, f"{bad} rows above {tol}, max rel {mx}"


def _from_lengths(lens, n, seed):
    """Rows with the given lengths (each at most n / 2): distinct sorted columns from a window
    of twice the row's length around the row, N(0,1) values."""
    rng = np.random.default_rng(seed)
    rows = []
    for r, L in enumerate(lens):
        span = min(n, 2 * L)
        lo = min(max(0, r - span // 2), n - span)
        rows.append(np.sort(lo + rng.choice(span, size=L, replace=False)))
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate(rows).astype(np.int32)
    v = rng.normal(size=int(rp[-1]))
    return M.from_arrays(len(lens), n, rp, ci, v)


CASES = {
    # rows of 2,000: 500 blocks per slice, many stages per slice
    "long_equal_rows": lambda: _from_lengths([2000] * 100, 50_000, 1),
    # empty slices between full ones, and at both ends
    "empty_slice_runs": lambda: _from_lengths(
        [0] * 64 + [9] * 32 + [0] * 96 + [7] * 40 + [0] * 33, 4_000, 2),
    # one row (a slice of one row and 31 absent ones: 4 nonzeros keep it within the
    # padding rule); 33 rows (a last slice of one row); 31 rows
    "one_row": lambda: _from_lengths([4], 100, 3),
    "thirty_three": lambda: _from_lengths([6] * 33, 200, 4),
    "thirty_one": lambda: _from_lengths([3] * 31, 200, 5),
    # far more slices than resident warps, short rows
    "many_slices": lambda: M.banded(400_000, 8, 5, seed=6),
    # a slice whose lengths differ inside a block (padding inside the last block only)
    "ragged_blocks": lambda: _from_lengths(list(np.arange(64) % 9 + 20), 5_000, 7),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("index_mode", [_abi.INDEX_I32, _abi.INDEX_AUTO], ids=["i32", "auto"])
def test_sell_shapes_fp64(cuda, name, index_mode):
    A = CASES[name]()
    assert M.sell_accepts(A)
    x = M.uniform(A.n, seed=11)
    y, info = _run(cuda, A, x, index_mode=index_mode)
    _check(y, A, x, 1e-12)
    assert info["format"] == _abi.FORMAT_SELL


@pytest.mark.parametrize("name", sorted(CASES))
def test_sell_shapes_fp32c(cuda, name):
    A = CASES[name]()
    A.v = A.v.astype(np.float32).astype(np.float64)
    x = M.uniform(A.n, seed=12, fp32=True)
    y, _ = _run(cuda, A, x, precision=_abi.PREC_FP32C, index_mode=_abi.INDEX_AUTO)
    _check(y, A, x, 1e-9)


def test_sell_16_bit_equals_32_bit_bitwise(cuda):
    """Per-slice base columns: the same sums, so the same bits."""
    A = M.banded(300_000, 64, 24, seed=8)
    x = M.uniform(A.n, seed=9)
    y32, i32 = _run(cuda, A, x, index_mode=_abi.INDEX_I32)
    y16, i16 = _run(cuda, A, x, index_mode=_abi.INDEX_DELTA16)
    assert i16["index_mode"] == _abi.INDEX_DELTA16 and i32["index_mode"] == _abi.INDEX_I32
    assert np.array_equal(y16, y32)


def test_sell_padding_threshold(cuda):
    """Accepted up to 2 nnz + 128 per slice stored elements, refused past it: one slice of 32
    rows, one of length L and 31 of length 1, stores 32 * ceil4(L) elements for L + 31 nonzeros,
    so L = 1..4 (128 stored) are taken and L = 5 (256 > 2 * 36 + 128) is refused."""
    def one_slice(L):
        return _from_lengths([L] + [1] * 31, 10_000, 13)
    ok = [L for L in range(1, 40) if M.sell_accepts(one_slice(L))]
    assert ok == [1, 2, 3, 4]
    for L in (max(ok), max(ok) + 1):
        A = one_slice(L)
        if M.sell_accepts(A):
            x = M.uniform(A.n, seed=14)
            y, _ = _run(cuda, A, x)
            _check(y, A, x, 1e-12)
        else:
            with pytest.raises(_abi.PavaError) as e:
                SpMatrix(A, "sell")
            assert e.value.status == _abi.E_UNSUPPORTED_PARAMS


def test_sell_empty_rows_ignore_nonfinite_x(cuda):
    """Padding and empty rows read no x: x is non-finite where no element reads it, and every
    row comes out finite, the empty ones exactly 0."""
    A = _from_lengths([0, 4, 0, 4, 3, 0, 4, 2] * 8, 500, 15)
    assert M.sell_accepts(A)
    read = np.zeros(A.n, bool)
    read[A.ci] = True
    x = M.uniform(A.n, seed=16)
    x[~read] = np.inf
    y, _ = _run(cuda, A, x)
    assert np.all(np.isfinite(y)) and np.all(y[np.diff(A.rp) == 0] == 0.0)
    _check(y, A, np.where(read, x, 0.0), 1e-12)


def _spmm_check(torch, A, k, tol, ldx_pad=0, **kw):
    """Y = A X on a SELL handle against the oracle, column by column; X row-major n x k with
    leading dimension k + ldx_pad."""
    fp32 = kw.get("precision") == _abi.PREC_FP32C
    Xh = M.uniform(A.n * (k + ldx_pad), seed=40 + k, fp32=fp32).reshape(A.n, k + ldx_pad)
    Xd = torch.from_numpy(Xh).to("cuda", torch.float32 if fp32 else torch.float64)[:, :k]
    mat = SpMatrix(A, "sell", **kw)
    Y = torch.full((A.m, k), float("nan"), dtype=torch.float64, device="cuda")
    mat.spmm(Xd, Y)
    Yh = Y.cpu().numpy()
    mat.close()
    for j in range(k):
        xj = np.ascontiguousarray(Xh[:, j])
        yr, ab = O.csr_ref(A.rp, A.ci, A.v, xj)
        bad, mx, _ = O.rel_error(np.ascontiguousarray(Yh[:, j]), yr, ab, tol)
        assert bad == 0, f"column {j}: {bad} rows above {tol}, max rel {mx}"


@pytest.mark.parametrize("k", [1, 3, 8, 16, 32, 33, 64])
@pytest.mark.parametrize("index_mode", [_abi.INDEX_I32, _abi.INDEX_AUTO], ids=["i32", "auto"])
def test_sell_spmm_fp64(cuda, k, index_mode):
    """Every k path: 1 column per lane (k <= 8), pairs of columns per read (even k up to 64),
    single columns (odd k); a banded matrix with some empty slices."""
    A = M.banded(20_000, 64, 24, seed=41)
    keep = np.ones(A.m, bool)
    keep[3_200:3_300] = False  # empty rows: three whole empty slices
    lens = np.where(keep, np.diff(A.rp), 0)
    sel = np.repeat(keep, np.diff(A.rp))
    B = M.from_arrays(A.m, A.n, np.concatenate([[0], np.cumsum(lens)]).astype(np.int32),
                      A.ci[sel], A.v[sel])
    assert M.sell_accepts(B)
    _spmm_check(cuda, B, k, 1e-12, index_mode=index_mode)


@pytest.mark.parametrize("k", [8, 32])
def test_sell_spmm_fp32c_and_strided_x(cuda, k):
    A = M.stencil27(20, seed=42)
    A.v = A.v.astype(np.float32).astype(np.float64)
    _spmm_check(cuda, A, k, 1e-9, precision=_abi.PREC_FP32C, index_mode=_abi.INDEX_AUTO)
    _spmm_check(cuda, A, k, 1e-12, ldx_pad=5)  # X with a leading dimension of k + 5


def test_sell_spmm_shapes(cuda):
    """Slices longer than a piece, ragged slices and empty-slice runs, k = 32."""
    for name in ("long_equal_rows", "empty_slice_runs", "thirty_three", "ragged_blocks"):
        _spmm_check(cuda, CASES[name](), 32, 1e-12)


def test_sell_spmm_k_limit(cuda):
    A = M.banded(2_000, 8, 5, seed=43)
    mat = SpMatrix(A, "sell")
    X = cuda.zeros((A.n, 65), dtype=cuda.float64, device="cuda")
    with pytest.raises(_abi.PavaError) as e:
        mat.spmm(X)
    assert e.value.status == _abi.E_UNSUPPORTED_PARAMS


@pytest.mark.parametrize("lanes,k", [(4, 1), (4, 5), (4, 8), (4, 16), (4, 27), (4, 32), (8, 8),
                                     (16, 16), (16, 31), (16, 64)])
def test_sell_spmm_lanes_per_row(cuda, lanes, k):
    """Every lanes-per-row shape the SpMM offers, even and odd k."""
    A = M.banded(10_000, 32, 12, seed=44)
    _spmm_check(cuda, A, k, 1e-12, lanes_per_row=lanes)


def test_sell_spmm_lanes_refused(cuda):
    A = M.banded(2_000, 8, 5, seed=45)
    with pytest.raises(_abi.PavaError) as e:
        SpMatrix(A, "sell", lanes_per_row=2)
    assert e.value.status == _abi.E_UNSUPPORTED_PARAMS
    mat = SpMatrix(A, "sell", lanes_per_row=4)
    X = cuda.zeros((A.n, 33), dtype=cuda.float64, device="cuda")
    with pytest.raises(_abi.PavaError) as e:
        mat.spmm(X)  # 4 lanes per row take k <= 32
    assert e.value.status == _abi.E_UNSUPPORTED_PARAMS
