"""The precision and index-compression forms against the FP64 oracle.

FP32C: values and x stored in FP32 (the matrices and x are drawn FP32-representable, so the
oracle's FP64 inputs are the exact widenings), FP32 compensated accumulation, FP64 carries.
Stated bound: relative error <= 1e-9 per row (cancellation-aware denominator).
DELTA16: 16-bit column offsets from a per-chunk base column; the arithmetic is unchanged, so
FP64 + DELTA16 must equal FP64 + I32 bit for bit."""
import numpy as np
import pytest

from oracle import oracle as O
from pava_b200 import _abi
from pava_b200 import matrices as M
from pava_b200.api import SpMatrix

pytestmark = pytest.mark.gpu

TOL32 = 1e-9
FORMS = [("cvr", dict(steps=64)), ("cvr", dict(steps=128)), ("csr5", dict(sigma=16)),
         ("csr5", dict(sigma=32, tiles_per_chunk=2)), ("sell", dict())]
FID = ["cvr64", "cvr128", "csr5s16", "csr5s32", "sell"]


def _refused(A, fmt, **kw):
    """True (after checking the refusal) where the SELL form must refuse A for its padding."""
    if fmt != "sell" or M.sell_accepts(A):
        return False
    with pytest.raises(_abi.PavaError) as e:
        SpMatrix(A, fmt, **kw)
    assert e.value.status == _abi.E_UNSUPPORTED_PARAMS
    return True


def _run(torch, A, x, fmt, precision, index_mode, **kw):
    mat = SpMatrix(A, fmt, precision=precision, index_mode=index_mode, **kw)
    dt = torch.float32 if precision == _abi.PREC_FP32C else torch.float64
    xd = torch.from_numpy(x).to("cuda", dt)
    y = torch.full((A.m,), float("nan"), dtype=torch.float64, device="cuda")
    mat.spmv(xd, y)
    return y.cpu().numpy(), mat


@pytest.mark.parametrize("fmt,kw", FORMS, ids=FID)
@pytest.mark.parametrize("index_mode", [_abi.INDEX_I32, _abi.INDEX_DELTA16], ids=["i32", "d16"])
def test_fp32c_stencil(cuda, fmt, kw, index_mode):
    A = M.stencil27(40, seed=2)
    x = M.uniform(A.n, seed=3, fp32=True)
    y, _ = _run(cuda, A, x, fmt, _abi.PREC_FP32C, index_mode, **kw)
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    bad, mx, mean = O.rel_error(y, yr, ab, TOL32)
    assert bad == 0, (mx, mean)
    # compensated accumulation is far better than the bound
    assert mx < 1e-12


@pytest.mark.parametrize("fmt,kw", FORMS, ids=FID)
def test_fp32c_irregular(cuda, fmt, kw):
    A = M.powerlaw(200_000, mean=16.0, cap=50_000, seed=5)
    A.v = A.v.astype(np.float32).astype(np.float64)
    x = M.uniform(A.n, seed=6, fp32=True)
    if _refused(A, fmt, precision=_abi.PREC_FP32C, **kw):
        return
    y, _ = _run(cuda, A, x, fmt, _abi.PREC_FP32C, _abi.INDEX_I32, **kw)
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    bad, mx, _ = O.rel_error(y, yr, ab, TOL32)
    assert bad == 0, mx


@pytest.mark.parametrize("fmt,kw", FORMS, ids=FID)
@pytest.mark.parametrize("index_mode", [_abi.INDEX_I32, _abi.INDEX_DELTA16], ids=["i32", "d16"])
def test_fp32c_empty_rows_between_full_chunks(cuda, fmt, kw, index_mode):
    # chunks with and without empty rows side by side (empty rows in two bands only); x is
    # non-finite where no element reads it: every empty row is exactly 0, every row finite
    A = M.stencil27(40, seed=11)
    lens = np.diff(A.rp)
    keep = np.ones(A.m, bool)
    keep[20_000:20_050] = False
    keep[41_000:41_003] = False
    keep[:5] = False
    rp = np.concatenate([[0], np.cumsum(np.where(keep, lens, 0))]).astype(np.int32)
    sel = np.repeat(keep, lens)
    B = M.from_arrays(A.m, A.n + 2, rp, A.ci[sel], A.v[sel].astype(np.float32).astype(np.float64))
    x = np.concatenate([M.uniform(A.n, seed=12, fp32=True), [np.inf, np.nan]])
    y, _ = _run(cuda, B, x, fmt, _abi.PREC_FP32C, index_mode, **kw)
    assert np.all(y[~keep] == 0.0) and np.all(np.isfinite(y))
    yr, ab = O.csr_ref(B.rp, B.ci, B.v, x)
    bad, mx, _ = O.rel_error(y, yr, ab, TOL32)
    assert bad == 0, mx


@pytest.mark.parametrize("fmt,kw", FORMS, ids=FID)
def test_fp64_delta16_equals_i32(cuda, fmt, kw):
    A = M.banded(300_000, 64, 24, seed=7)
    x = M.uniform(A.n, seed=8)
    y32, _ = _run(cuda, A, x, fmt, _abi.PREC_FP64, _abi.INDEX_I32, **kw)
    y16, _ = _run(cuda, A, x, fmt, _abi.PREC_FP64, _abi.INDEX_DELTA16, **kw)
    assert np.array_equal(y32, y16)
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    assert O.rel_error(y16, yr, ab, 1e-12)[0] == 0


def test_delta16_out_of_range_rejected(cuda):
    # random columns over 200,000: every chunk spans far more than 65,534 columns
    A = M.random_csr(50_000, 200_000, 8.0, seed=9)
    with pytest.raises(_abi.PavaError) as e:
        SpMatrix(A, "cvr", index_mode=_abi.INDEX_DELTA16)
    assert e.value.status == _abi.E_UNSUPPORTED_PARAMS


def test_fp32c_wrong_x_dtype_rejected(cuda):
    A = M.laplace2d(32)
    mat = SpMatrix(A, "cvr", precision=_abi.PREC_FP32C)
    with pytest.raises(TypeError):
        mat.spmv(cuda.zeros(A.n, dtype=cuda.float64, device="cuda"))


def test_config3_full_size_fp32c_vs_fp64(cuda):
    """128^3 27-point stencil: FP64 drop-in within 1e-12, FP32C within 1e-9 of the oracle."""
    A = M.stencil27(128, seed=2)
    x = M.uniform(A.n, seed=3, fp32=True)
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    y64, m64 = _run(cuda, A, x, "csr5", _abi.PREC_FP64, _abi.INDEX_I32)
    assert O.rel_error(y64, yr, ab, 1e-12)[0] == 0
    del m64
    for fmt in ("cvr", "csr5", "sell"):
        y32, m32 = _run(cuda, A, x, fmt, _abi.PREC_FP32C, _abi.INDEX_DELTA16)
        bad, mx, mean = O.rel_error(y32, yr, ab, TOL32)
        assert bad == 0, (fmt, mx, mean)
        del m32


@pytest.mark.parametrize("fmt,kw", FORMS, ids=FID)
def test_delta16_reaches_any_chunk_of_narrow_column_span(cuda, fmt, kw):
    """16-bit offsets are taken from each chunk's base column (the middle of its column
    range): a random 40,000 x 40,000 matrix has columns up to 39,999 away from their row but
    every chunk spans fewer than 65,535 columns, so it converts with 16-bit offsets; FP64
    results are bitwise those of 32-bit columns, FP32C within its bound."""
    torch = cuda
    A = M.random_csr(40_000, 40_000, 9.0, seed=12)
    x = M.uniform(A.n, seed=13, fp32=True)
    A.v = A.v.astype(np.float32).astype(np.float64)
    xd = torch.from_numpy(x).cuda()
    d16 = SpMatrix(A, fmt, index_mode=_abi.INDEX_DELTA16, **kw)
    assert d16.info()["index_mode"] == _abi.INDEX_DELTA16
    y16 = d16.spmv(xd).cpu().numpy()
    y32 = SpMatrix(A, fmt, index_mode=_abi.INDEX_I32, **kw).spmv(xd).cpu().numpy()
    assert np.array_equal(y16, y32)
    y, _ = _run(torch, A, x, fmt, _abi.PREC_FP32C, _abi.INDEX_AUTO, **kw)
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    assert O.rel_error(y, yr, ab, TOL32)[0] == 0


@pytest.mark.parametrize("fmt,kw", FORMS, ids=FID)
def test_delta16_span_limit(cuda, fmt, kw):
    """Every row reads the first and the last column, so every chunk spans n - 1 columns:
    n = 65,535 (span 65,534) fits 16-bit offsets, n = 65,536 does not."""
    torch = cuda
    rng = np.random.default_rng(14)
    for n, fits in ((65_535, True), (65_536, False)):
        m = 3_000
        cols = [np.unique(np.concatenate([[0, n - 1], rng.integers(1, n - 1, 6)])) for _ in range(m)]
        rp = np.concatenate([[0], np.cumsum([len(c) for c in cols])]).astype(np.int32)
        ci = np.concatenate(cols).astype(np.int32)
        A = M.from_arrays(m, n, rp, ci, rng.normal(size=len(ci)))
        if not fits:
            with pytest.raises(_abi.PavaError) as e:
                SpMatrix(A, fmt, index_mode=_abi.INDEX_DELTA16, **kw)
            assert e.value.status == _abi.E_UNSUPPORTED_PARAMS
            assert SpMatrix(A, fmt, index_mode=_abi.INDEX_AUTO, **kw).info()["index_mode"] == \
                _abi.INDEX_I32
            continue
        xd = torch.from_numpy(M.uniform(n, seed=15)).cuda()
        d16 = SpMatrix(A, fmt, index_mode=_abi.INDEX_DELTA16, **kw)
        y16 = d16.spmv(xd).cpu().numpy()
        y32 = SpMatrix(A, fmt, index_mode=_abi.INDEX_I32, **kw).spmv(xd).cpu().numpy()
        assert np.array_equal(y16, y32)
        yr, ab = O.csr_ref(A.rp, A.ci, A.v, xd.cpu().numpy())
        assert O.rel_error(y16, yr, ab, 1e-12)[0] == 0


@pytest.mark.parametrize("fmt,kw", FORMS, ids=FID)
def test_index_auto_picks_16_bit_where_it_fits(cuda, fmt, kw):
    """PAVA_INDEX_AUTO: 16-bit offsets on a stencil, 32-bit columns when a column is out of
    reach; results bitwise equal to the 32-bit form either way."""
    torch = cuda
    for A, want in ((M.stencil27(30, seed=9), _abi.INDEX_DELTA16),
                    (M.powerlaw(300_000, mean=12.0, seed=10), _abi.INDEX_I32),
                    (M.random_csr(30_000, 300_000, 6.0, seed=16), _abi.INDEX_I32)):
        if _refused(A, fmt, index_mode=_abi.INDEX_AUTO, **kw):
            continue
        x = torch.from_numpy(M.uniform(A.n, seed=11)).cuda()
        auto = SpMatrix(A, fmt, index_mode=_abi.INDEX_AUTO, **kw)
        assert auto.info()["index_mode"] == want
        y_auto = auto.spmv(x).cpu().numpy()
        y_i32 = SpMatrix(A, fmt, index_mode=_abi.INDEX_I32, **kw).spmv(x).cpu().numpy()
        assert np.array_equal(y_auto, y_i32)
