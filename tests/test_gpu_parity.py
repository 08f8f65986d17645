"""Parity of the CUDA engine (through the C ABI) with the oracle: the long-double CSR product
and the restated reference CVR / CSR5 engines, on the golden fixtures, the benchmark
configurations at full size, and edge cases.  The SELL form converts exactly the matrices whose
slice padding at most doubles the stored elements (matrices.sell_accepts) and refuses the rest
with PAVA_E_UNSUPPORTED_PARAMS; every test checks one or the other.

Tolerance (FP64 drop-in): 1e-12 relative per row, with the cancellation-aware denominator
max(|y_ref_i|, sum_j |a_ij x_j|)."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from pava_b200 import _abi
from pava_b200 import matrices as M
from pava_b200.api import AnonymousLibHandle, SpMatrix, conduct_csr5, conduct_cvr

pytestmark = pytest.mark.gpu

TOL = 1e-12
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))

VARIANTS = [("cvr", dict(steps=32)), ("cvr", dict(steps=64)), ("cvr", dict(steps=128)),
            ("csr5", dict(sigma=16, tiles_per_chunk=4)), ("csr5", dict(sigma=8, tiles_per_chunk=1)),
            ("csr5", dict(sigma=32, tiles_per_chunk=2)), ("csr5", dict(sigma=12, tiles_per_chunk=3)),
            ("csr", dict()), ("sell", dict())]
VID = [f"{f}-" + "-".join(f"{k}{v}" for k, v in kw.items()) for f, kw in VARIANTS]
# the forms with a per-chunk 16-bit column base (all but plain CSR)
D16_VARIANTS = [v for v in VARIANTS if v[0] != "csr"]
D16_VID = [i for v, i in zip(VARIANTS, VID) if v[0] != "csr"]


def _gpu_y(torch, A, x, fmt, **kw):
    """(y, handle) of one SpMV, or (None, None) where the SELL form refuses A as it must."""
    if fmt == "sell" and not M.sell_accepts(A):
        with pytest.raises(_abi.PavaError) as e:
            SpMatrix(A, fmt, **kw)
        assert e.value.status == _abi.E_UNSUPPORTED_PARAMS and "padding" in str(e.value)
        return None, None
    mat = SpMatrix(A, fmt, **kw)
    xd = torch.from_numpy(x).cuda()
    y = torch.full((A.m,), float("nan"), dtype=torch.float64, device="cuda")
    mat.spmv(xd, y)
    y1 = y.cpu().numpy().copy()
    mat.spmv(xd, y)
    y2 = y.cpu().numpy()
    assert np.array_equal(y1, y2, equal_nan=True), "repeated SpMV differs"
    return y1, mat


def _check(y, A, x, tol=TOL):
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    bad, mx, _ = O.rel_error(y, yr, ab, tol)
    assert bad == 0, f"{bad} rows above {tol}, max rel {mx}"
    return yr, ab


@pytest.mark.parametrize("fmt,kw", VARIANTS, ids=VID)
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_golden(cuda, path, fmt, kw):
    d = np.load(path)
    A = M.from_arrays(d["m"], d["n"], d["rp"], d["ci"], d["v"])
    x = d["x"]
    y, _ = _gpu_y(cuda, A, x, fmt, **kw)
    if y is None:
        return
    yr, ab = _check(y, A, x)
    # against the reference's own CVR and CSR5 outputs stored in the fixture
    for key in ("y_cvr", "y_csr5"):
        assert O.rel_error(y, d[key], ab, TOL)[0] == 0


def test_laplace512_full_size_vs_reference_cvr(cuda):
    A = M.laplace2d(512)
    x = M.uniform(A.n, seed=0)
    y_port, _, _ = O.cvr_port(A.rp, A.ci, A.v, x, nthreads=8)
    for fmt, kw in VARIANTS:
        y, _ = _gpu_y(cuda, A, x, fmt, **kw)
        assert y is not None
        yr, ab = _check(y, A, x)
        assert O.rel_error(y, y_port, ab, TOL)[0] == 0
        # rows a single lane sums are bit-identical to a sequential FMA sum; the 5-point rows
        # never split in CVR, so CVR equals the reference CVR exactly on this matrix, and SELL
        # sums every row in one lane
        if fmt in ("cvr", "sell"):
            assert np.max(np.abs(y - y_port)) <= 4.5e-16 * 8


@pytest.mark.parametrize("fmt,kw", VARIANTS[:4] + VARIANTS[7:], ids=VID[:4] + VID[7:])
def test_powerlaw_long_rows(cuda, fmt, kw):
    # rows up to 60,000 nnz span many chunks; 2 % empty rows
    A = M.powerlaw(200_000, mean=16.0, sigma=2.0, cap=60_000, seed=21)
    x = M.uniform(A.n, seed=22)
    y, _ = _gpu_y(cuda, A, x, fmt, **kw)
    if y is None:
        return
    yr, ab = _check(y, A, x)
    y_csr5, _, _ = O.csr5_port(A.rp, A.ci, A.v, x, nthreads=8)
    assert O.rel_error(y, y_csr5, ab, TOL)[0] == 0


def _edge_cases():
    out = []
    # single row
    out.append(("one_row", M.from_arrays(1, 10, [0, 3], [1, 4, 9], [1.0, -2.0, 0.5])))
    # all rows empty
    out.append(("all_empty", M.from_arrays(100, 100, np.zeros(101, np.int32), [], [])))
    # leading/trailing empty rows and a long row across chunks
    L = 10_000
    rp = np.array([0, 0, 0, L, L + 1, L + 1, L + 3, L + 3], np.int32)
    ci = np.concatenate([np.arange(L) % 7000, [5, 6, 7]]).astype(np.int32)
    ci[:L] = np.sort(np.random.default_rng(1).choice(7000, L, replace=True))
    v = np.random.default_rng(2).normal(size=L + 3)
    out.append(("long_row_empties", M.from_arrays(7, 7000, rp, ci, v)))
    # exactly one chunk of elements, many 1-element rows
    out.append(("ones_2048", M.from_arrays(2048, 2048, np.arange(2049, dtype=np.int32),
                                           np.arange(2048, dtype=np.int32), np.ones(2048))))
    # wide matrix, n != m
    out.append(("wide", M.random_csr(3000, 500_000, 40.0, seed=8)))
    out.append(("tall", M.random_csr(200_000, 50, 3.0, seed=9)))
    # 90 % empty rows
    out.append(("mostly_empty", M.powerlaw(50_000, mean=8.0, p_empty=0.9, seed=10)))
    # rows of exactly 32*S elements at chunk boundaries
    rp = np.arange(0, 2048 * 6 + 1, 2048, dtype=np.int32)
    out.append(("chunk_rows", M.from_arrays(6, 2048, rp, np.tile(np.arange(2048), 6).astype(np.int32),
                                            np.random.default_rng(3).normal(size=2048 * 6))))
    return out


EDGE = _edge_cases()


@pytest.mark.parametrize("fmt,kw", VARIANTS, ids=VID)
@pytest.mark.parametrize("name,A", EDGE, ids=[e[0] for e in EDGE])
def test_edge_cases(cuda, name, A, fmt, kw):
    x = M.uniform(A.n, seed=31)
    y, _ = _gpu_y(cuda, A, x, fmt, **kw)
    if y is not None:
        _check(y, A, x)


@pytest.mark.parametrize("fmt,kw", D16_VARIANTS, ids=D16_VID)
@pytest.mark.parametrize("name,A", EDGE, ids=[e[0] for e in EDGE])
def test_edge_cases_16_bit_offsets(cuda, name, A, fmt, kw):
    """The edge cases with PAVA_INDEX_AUTO (16-bit offsets from each chunk's base column where
    they reach: empty and all-padding chunks, rows across chunks): bitwise the 32-bit form."""
    x = M.uniform(A.n, seed=32)
    y16, mat = _gpu_y(cuda, A, x, fmt, index_mode=_abi.INDEX_AUTO, **kw)
    y32, _ = _gpu_y(cuda, A, x, fmt, **kw)
    if y16 is None:
        return
    assert np.array_equal(y16, y32)
    if A.n <= 65_535:  # every chunk's columns fit a 65,534 span
        assert mat.info()["index_mode"] == _abi.INDEX_DELTA16


def test_empty_rows_are_zero_even_with_nonfinite_x(cuda):
    A = M.from_arrays(4, 3, [0, 1, 1, 2, 2], [0, 2], [2.0, 3.0])
    x = np.array([1.0, np.inf, 2.0])
    for fmt in ("cvr", "csr5", "sell"):
        y, _ = _gpu_y(cuda, A, x, fmt)
        assert y[1] == 0.0 and y[3] == 0.0 and y[0] == 2.0 and y[2] == 6.0


def test_host_entry_point_matches_device(cuda):
    for A in (M.powerlaw(100_000, seed=41), M.stencil27(40, seed=4)):
        x = M.uniform(A.n, seed=42)
        for fmt in ("cvr", "csr5", "csr", "sell"):
            y, mat = _gpu_y(cuda, A, x, fmt)
            if y is None:
                continue
            yh = mat.spmv_host(x)
            assert np.array_equal(yh, y)


def test_invalid_csr_rejected(cuda):
    bad = M.from_arrays(3, 3, [0, 2, 1, 3], [0, 1, 2], [1.0, 1.0, 1.0])
    with pytest.raises(_abi.PavaError) as e:
        SpMatrix(bad, "cvr")
    assert e.value.status == _abi.E_INVALID_CSR
    badcol = M.from_arrays(2, 3, [0, 1, 2], [0, 3], [1.0, 1.0])
    with pytest.raises(_abi.PavaError) as e:
        SpMatrix(badcol, "csr5")
    assert e.value.status == _abi.E_INVALID_CSR


def test_bad_parameters_rejected(cuda):
    A = M.laplace2d(16)
    with pytest.raises(_abi.PavaError) as e:
        SpMatrix(A, "cvr", steps=48)
    assert e.value.status == _abi.E_UNSUPPORTED_PARAMS
    with pytest.raises(_abi.PavaError) as e:
        SpMatrix(A, "csr5", sigma=10)
    assert e.value.status == _abi.E_UNSUPPORTED_PARAMS


def test_conduct_entry_points(cuda, capfd):
    A = M.laplace2d(128)
    x, y, _ = M.init_vectors(A.m, A.n)  # x[i] = i % 3, as the reference benchmark
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    out = np.zeros(A.m)
    assert conduct_cvr(A.m, A.n, A.nnz, A.rp, A.ci, A.v, x, out, 1, "Syn lap128", 20) == 0
    assert O.rel_error(out, yr, ab, TOL)[0] == 0 and O.check_results(out, yr) == 0
    out2 = np.zeros(A.m)
    assert conduct_csr5(A.m, A.n, A.nnz, A.rp, A.ci, A.v, x, out2, 1.0, "Syn lap128", 20) == 0
    assert O.rel_error(out2, yr, ab, TOL)[0] == 0
    lines = [ln for ln in capfd.readouterr().out.splitlines() if ln.startswith(" Performance")]
    assert len(lines) == 2
    f = lines[0].split()
    assert f[1:4] == ["Syn", "lap128", "CVR"] and float(f[5]) > 0 and float(f[6]) > 0


def test_anonymouslib_handle_contract(cuda):
    A = M.powerlaw(20_000, seed=51)
    x = M.uniform(A.n, seed=52)
    h = AnonymousLibHandle(A.m, A.n)
    y = np.zeros(A.m)
    assert h.inputCSR(A.nnz, A.rp, A.ci, A.v) == 0
    assert h.setX(x) == 0
    assert h.spmv(1.0, y) == -4  # ANONYMOUSLIB_UNSUPPORTED_CSR_SPMV before asCSR5
    h.setSigma(16)
    assert h.asCSR5() == 0
    assert h.spmv(1.0, y) == 0
    _check(y, A, x)
    y2 = np.zeros(A.m)
    assert h.spmv(1.0, y2) == 0 and np.array_equal(y, y2)  # no accumulation across calls
    assert h.asCSR() == 0 and h.destroy() == 0
    h2 = AnonymousLibHandle(A.m, A.n)
    h2.inputCSR(A.nnz, A.rp, A.ci, A.v)
    h2.setSigma(10)
    assert h2.asCSR5() == -2  # ANONYMOUSLIB_UNSUPPORTED_CSR5_OMEGA


def test_config2_full_size(cuda):
    """The 4,194,304-row power-law matrix (~64 M nnz) of the headline benchmark."""
    A = M.powerlaw(4_194_304, seed=1)
    x = M.uniform(A.n, seed=1)
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    ys = []
    for fmt in ("cvr", "csr5"):
        y, mat = _gpu_y(cuda, A, x, fmt)
        bad, mx, mean = O.rel_error(y, yr, ab, TOL)
        assert bad == 0, (fmt, mx)
        ys.append(y)
        del mat
    # size-independent property: the two formats agree with each other row by row
    assert O.rel_error(ys[0], ys[1], ab, 2 * TOL)[0] == 0


@pytest.mark.parametrize("fmt", ["cvr", "csr5", "csr", "sell"])
def test_memory_budget_gives_nomem_and_frees(cuda, fmt):
    """A handle whose arrays would pass the device memory budget fails with PAVA_E_NOMEM and
    leaves no device memory behind; without the budget the same matrix converts."""
    torch = cuda
    L = _abi.gpu()
    A = M.stencil27(40, seed=61) if fmt == "sell" else M.powerlaw(200_000, seed=61)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    try:
        assert L.pava_set_device_memory_limit(1 << 20) == 0
        with pytest.raises(_abi.PavaError) as e:
            SpMatrix(A, fmt)
        assert e.value.status == _abi.E_NOMEM
    finally:
        L.pava_set_device_memory_limit(0)
    torch.cuda.synchronize()
    assert abs(torch.cuda.mem_get_info()[0] - free0) < (8 << 20)
    mat = SpMatrix(A, fmt)
    assert mat.info()["device_bytes"] > (1 << 20)
    mat.close()
