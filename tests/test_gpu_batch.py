"""Multi-RHS products, batches of independent matrices, graph replay and the autotuner,
through the C ABI, against the CPU oracle (long-double CSR sums).

Bounds: FP64 forms 1e-12 relative per row and right-hand side (cancellation-aware
denominator); FP32C forms 1e-9 on FP32-representable inputs."""
import numpy as np
import pytest

from oracle import oracle as O
from pava_b200 import _abi
from pava_b200 import matrices as M
from pava_b200.api import Batch, SpMatrix, autotune

pytestmark = pytest.mark.gpu

TOL = 1e-12
TOL32 = 1e-9


def _check_cols(A, X, Y, tol):
    for j in range(X.shape[1]):
        yr, ab = O.csr_ref(A.rp, A.ci, A.v, np.ascontiguousarray(X[:, j]))
        bad, mx, _ = O.rel_error(np.ascontiguousarray(Y[:, j]), yr, ab, tol)
        assert bad == 0, (j, mx)


def _x(torch, n, k, seed, fp32=False):
    X = M.uniform(n * k, seed=seed, fp32=fp32).reshape(n, k)
    return X, torch.from_numpy(X).to("cuda", torch.float32 if fp32 else torch.float64)


SHAPES = [  # (k, lanes_per_row, col_lanes, cols_per_lane, rows_per_tile)
    (1, 0, 0, 0, 0), (1, 4, 1, 1, 64), (1, 32, 1, 1, 1), (2, 8, 2, 1, 0), (8, 8, 8, 1, 4),
    (8, 32, 8, 1, 0), (8, 16, 4, 2, 0), (13, 16, 16, 1, 2), (32, 32, 32, 1, 0),
    (32, 32, 16, 2, 3), (32, 16, 8, 4, 0), (64, 32, 32, 2, 0), (100, 32, 32, 4, 1),
]


@pytest.mark.parametrize("k,gl,kc,kpl,tr", SHAPES, ids=[f"k{s[0]}_g{s[1]}_c{s[2]}_p{s[3]}_t{s[4]}" for s in SHAPES])
def test_spmm_banded_shapes(cuda, k, gl, kc, kpl, tr):
    torch = cuda
    A = M.banded(20_000, 64, 24, seed=11)
    X, Xd = _x(torch, A.n, k, seed=12)
    mat = SpMatrix(A, "csr", lanes_per_row=gl, col_lanes=kc, cols_per_lane=kpl, rows_per_tile=tr)
    Y = mat.spmm(Xd).cpu().numpy()
    _check_cols(A, X, Y, TOL)


WINDOW = [  # (k, lanes_per_row, col_lanes, cols_per_lane, rows_per_tile)
    (8, 8, 8, 1, 0), (8, 8, 4, 2, 32), (32, 32, 32, 1, 8), (32, 8, 8, 4, 128),
    (13, 16, 16, 1, 0), (2, 4, 2, 1, 256), (64, 32, 32, 2, 0),
]


@pytest.mark.parametrize("k,gl,kc,kpl,tr", WINDOW, ids=[f"k{s[0]}_g{s[1]}_c{s[2]}_p{s[3]}_t{s[4]}" for s in WINDOW])
def test_spmm_x_window(cuda, k, gl, kc, kpl, tr):
    """X windows staged in shared memory: banded rows (every tile staged), power-law rows
    (wide windows: the global-gather fallback) and a ragged last tile."""
    torch = cuda
    for A in (M.banded(20_003, 64, 24, seed=31), M.powerlaw(9_001, mean=10.0, p_empty=0.05, seed=32)):
        X, Xd = _x(torch, A.n, k, seed=33)
        mat = SpMatrix(A, "csr", lanes_per_row=gl, col_lanes=kc, cols_per_lane=kpl,
                       rows_per_tile=tr, x_window=1)
        Y = mat.spmm(Xd).cpu().numpy()
        _check_cols(A, X, Y, TOL)
        # the same arithmetic order as the global-gather kernel: identical bits
        ref = SpMatrix(A, "csr", lanes_per_row=gl, col_lanes=kc, cols_per_lane=kpl).spmm(Xd)
        assert np.array_equal(Y, ref.cpu().numpy())


def test_spmm_x_window_fp32c(cuda):
    torch = cuda
    A = M.stencil27(24, seed=34)
    X, Xd = _x(torch, A.n, 16, seed=35, fp32=True)
    mat = SpMatrix(A, "csr", precision=_abi.PREC_FP32C, lanes_per_row=16, col_lanes=16,
                   x_window=1)
    _check_cols(A, X, mat.spmm(Xd).cpu().numpy(), TOL32)


def test_spmm_irregular_rows_and_strides(cuda):
    torch = cuda
    A = M.powerlaw(30_000, mean=16.0, cap=5_000, p_empty=0.05, seed=13)
    X, Xd = _x(torch, A.n, 24, seed=14)
    # X and Y as column slices of wider row-major buffers (ldx, ldy > k)
    Xw = torch.zeros((A.n, 40), dtype=torch.float64, device="cuda")
    Xw[:, 3:27] = Xd
    Yw = torch.full((A.m, 33), float("nan"), dtype=torch.float64, device="cuda")
    mat = SpMatrix(A, "csr", lanes_per_row=32, col_lanes=8, cols_per_lane=4)
    mat.spmm(Xw[:, 3:27], Yw[:, 5:29])
    Y = Yw[:, 5:29].cpu().numpy()
    _check_cols(A, X, Y, TOL)
    assert torch.isnan(Yw[:, :5]).all() and torch.isnan(Yw[:, 29:]).all()


def test_spmm_k1_equals_spmv(cuda):
    torch = cuda
    A = M.random_csr(50_000, mean=12.0, seed=15)
    x = M.uniform(A.n, seed=16)
    mat = SpMatrix(A, "csr", lanes_per_row=4)
    y1 = mat.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
    y2 = mat.spmm(torch.from_numpy(x).cuda().reshape(-1, 1)).cpu().numpy()[:, 0]
    assert np.array_equal(y1, y2)


def test_spmm_fp32c(cuda):
    torch = cuda
    A = M.stencil27(24, seed=17)
    X, Xd = _x(torch, A.n, 8, seed=18, fp32=True)
    mat = SpMatrix(A, "csr", precision=_abi.PREC_FP32C, lanes_per_row=8, col_lanes=8)
    Y = mat.spmm(Xd).cpu().numpy()
    _check_cols(A, X, Y, TOL32)


@pytest.mark.parametrize("kw", [dict(lanes_per_row=3), dict(col_lanes=64),
                                dict(cols_per_lane=3), dict(lanes_per_row=4, col_lanes=8),
                                dict(lanes_per_row=4, rows_per_tile=3),
                                dict(lanes_per_row=8, rows_per_tile=8, x_window=1)],
                         ids=["gl3", "kc64", "kpl3", "kc_gt_gl", "tr_not_multiple",
                              "window_tr_not_multiple"])
def test_csr_shape_rejected(cuda, kw):
    A = M.random_csr(1000, seed=19)
    with pytest.raises(_abi.PavaError) as e:
        SpMatrix(A, "csr", **kw)
    assert e.value.status == _abi.E_UNSUPPORTED_PARAMS


def test_spmm_k_not_covered(cuda):
    torch = cuda
    A = M.random_csr(1000, seed=20)
    mat = SpMatrix(A, "csr", col_lanes=4, cols_per_lane=2)
    Xd = torch.zeros((A.n, 9), dtype=torch.float64, device="cuda")
    with pytest.raises(_abi.PavaError) as e:
        mat.spmm(Xd)
    assert e.value.status == _abi.E_UNSUPPORTED_PARAMS


# ---- batches ------------------------------------------------------------------------------

def _batch_mats(count, seed, lo=64, hi=6000):
    rng = np.random.default_rng(seed)
    mats = []
    for i in range(count):
        m = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        mats.append(M.random_csr(m, mean=12.0, seed=seed * 1000 + i))
    # uneven extras: an all-empty matrix, one with empty rows, a rectangular one, 1 x 1
    mats.append(M.from_arrays(40, 40, np.zeros(41, np.int32), [], []))
    mats.append(M.powerlaw(3000, mean=4.0, p_empty=0.3, seed=seed + 1))
    mats.append(M.random_csr(700, n=1900, mean=9.0, seed=seed + 2))
    mats.append(M.from_arrays(1, 1, [0, 1], [0], [2.5]))
    return mats


def _check_batch(b, mats, xs, y, tol):
    for i, A in enumerate(mats):
        yi = y[b.y_offsets[i]: b.y_offsets[i + 1]]
        yr, ab = O.csr_ref(A.rp, A.ci, A.v, xs[i])
        bad, mx, _ = O.rel_error(yi, yr, ab, tol)
        assert bad == 0, (i, mx)


BATCH_FORMS = [("csr", dict(lanes_per_row=4)), ("csr", dict(lanes_per_row=16, rows_per_tile=32)),
               ("cvr", dict(steps=64)), ("csr5", dict(sigma=16)), ("auto", {})]


@pytest.mark.parametrize("fmt,kw", BATCH_FORMS, ids=["csr4", "csr16", "cvr", "csr5", "auto"])
def test_batch_matches_each_matrix(cuda, fmt, kw):
    torch = cuda
    mats = _batch_mats(60, seed=21)
    b = Batch(mats, fmt, **kw)
    assert b.count == len(mats) and b.m == sum(A.m for A in mats)
    xs = [M.uniform(A.n, seed=100 + i) for i, A in enumerate(mats)]
    x = torch.from_numpy(np.concatenate(xs)).cuda()
    y = b.spmv(x).cpu().numpy()
    _check_batch(b, mats, xs, y, TOL)
    if fmt == "auto":
        f, o = b.chosen()
        assert f in ("csr", "cvr", "csr5")


def test_batch_graph_replay_bitwise(cuda):
    torch = cuda
    mats = _batch_mats(40, seed=22)
    b = Batch(mats, "csr", lanes_per_row=4)
    xs = [M.uniform(A.n, seed=200 + i) for i, A in enumerate(mats)]
    x = torch.from_numpy(np.concatenate(xs)).cuda()
    y_direct = b.spmv(x).cpu().numpy()
    y = torch.full((b.m,), float("nan"), dtype=torch.float64, device="cuda")
    b.capture(x, y)
    for _ in range(3):
        y.fill_(float("nan"))
        b.replay()
        torch.cuda.synchronize()
        assert np.array_equal(y.cpu().numpy(), y_direct)
    # the graph reads x at replay time: new x values, same buffer
    xs2 = [M.uniform(A.n, seed=300 + i) for i, A in enumerate(mats)]
    x.copy_(torch.from_numpy(np.concatenate(xs2)))
    b.replay()
    torch.cuda.synchronize()
    _check_batch(b, mats, xs2, y.cpu().numpy(), TOL)


def test_batch_fp32c(cuda):
    torch = cuda
    mats = [M.stencil27(g, seed=23 + g) for g in (6, 9, 13)] + _batch_mats(10, seed=24)
    for A in mats:
        A.v = A.v.astype(np.float32).astype(np.float64)
    xs = [M.uniform(A.n, seed=400 + i, fp32=True) for i, A in enumerate(mats)]
    for fmt, kw in [("csr", dict(lanes_per_row=8)), ("csr5", dict(sigma=32))]:
        b = Batch(mats, fmt, precision=_abi.PREC_FP32C, **kw)
        x = torch.from_numpy(np.concatenate(xs)).to("cuda", torch.float32)
        y = b.spmv(x).cpu().numpy()
        _check_batch(b, mats, xs, y, TOL32)


def test_batch_rejects_bad_matrix(cuda):
    mats = _batch_mats(5, seed=25)
    bad = M.random_csr(100, seed=26)
    bad.ci = bad.ci.copy()
    bad.ci[7] = 100  # column == n
    with pytest.raises(_abi.PavaError) as e:
        Batch(mats + [bad], "csr")
    assert e.value.status == _abi.E_INVALID_CSR
    norows = M.from_arrays(0, 5, [0], [], [])
    norows.rp = np.array([3], np.int32)  # claims 3 nonzeros with no rows
    norows.ci = np.zeros(3, np.int32)
    norows.v = np.ones(3)
    with pytest.raises(_abi.PavaError) as e:
        Batch(mats + [norows], "csr")
    assert e.value.status == _abi.E_INVALID_CSR


# ---- autotuner ----------------------------------------------------------------------------

def test_autotune_k1_runs_every_candidate(cuda):
    A = M.powerlaw(100_000, mean=16.0, cap=20_000, seed=27)
    ents, best = autotune(A, k=1, reps=3)
    forms = {e["format"] for e in ents}
    assert {"cvr", "csr5", "csr", "sell"} <= forms
    # CVR / CSR5 / SELL come with 32-bit columns and with 16-bit offsets where they reach
    modes = {(e["format"], e["opts"]["index_mode"]) for e in ents if e["format"] != "csr"}
    assert modes == {(f, m) for f in ("cvr", "csr5", "sell")
                     for m in (_abi.INDEX_I32, _abi.INDEX_AUTO)}
    # SELL refuses the power-law rows (its padding would be ~10x); every other form runs
    assert not M.sell_accepts(A)
    for e in ents:
        if e["format"] == "sell":
            assert e["status"] == _abi.E_UNSUPPORTED_PARAMS and e["ms"] < 0
        else:
            assert e["ms"] > 0 and e["status"] == 0
    assert ents[best]["ms"] == min(e["ms"] for e in ents if e["ms"] > 0)
    # the winner computes the right product
    torch = cuda
    x = M.uniform(A.n, seed=28)
    e = ents[best]
    opts = {k: v for k, v in e["opts"].items() if v and k != "precision"}
    y = SpMatrix(A, e["format"], **opts).spmv(torch.from_numpy(x).cuda()).cpu().numpy()
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    assert O.rel_error(y, yr, ab, TOL)[0] == 0


def test_autotune_wave_balanced_csr5(cuda):
    """CSR5 candidates come with the default tiles per chunk and with PAVA_TILES_WAVE, the
    count that fills the last wave of warp chunks (24 resident warps per SM): on the
    1,048,576-row banded matrix, sigma 32 has 24,576 tiles; 7 per chunk make 3,511 chunks, one
    wave on 148 SMs.  A wave form whose count equals the default is timed once."""
    torch = cuda
    A = M.banded(1_048_576, 64, 24, seed=3)
    warps = 24 * torch.cuda.get_device_properties(0).multi_processor_count

    def wave(tiles):  # fewest tiles on a warp's critical path, the largest G among equals
        return min(range(1, 9), key=lambda g: (-(-tiles // (g * warps)) * g, -g))

    def default(tiles):
        return 4 if tiles >= 4 * warps else (2 if tiles >= 2 * warps else 1)

    ents, best = autotune(A, k=1, reps=2)
    assert len(ents) == _abi.NVARIANTS
    for sg in (16, 32):
        tiles = A.nnz // (32 * sg)
        es = [e for e in ents if e["format"] == "csr5" and e["opts"]["sigma"] == sg]
        assert {e["opts"]["tiles_per_chunk"] for e in es} == {0, _abi.TILES_WAVE}
        for tpc in (0, _abi.TILES_WAVE):
            g = wave(tiles) if tpc == _abi.TILES_WAVE else default(tiles)
            mat = SpMatrix(A, "csr5", sigma=sg, tiles_per_chunk=tpc)
            assert mat.info()["elems_per_chunk"] == 32 * sg * g
            mat.close()
        if wave(tiles) == default(tiles):  # the same form: one timing for both entries
            d = {e["opts"]["tiles_per_chunk"]: e["ms"] for e in es
                 if e["opts"]["index_mode"] == _abi.INDEX_I32}
            assert d[0] == d[_abi.TILES_WAVE]
    # the wave-balanced form computes the same product as the default one
    x = torch.from_numpy(M.uniform(A.n, seed=33)).cuda()
    y0 = SpMatrix(A, "csr5", sigma=32).spmv(x).cpu().numpy()
    y1 = SpMatrix(A, "csr5", sigma=32, tiles_per_chunk=_abi.TILES_WAVE).spmv(x).cpu().numpy()
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x.cpu().numpy())
    assert O.rel_error(y0, yr, ab, TOL)[0] == 0 and O.rel_error(y1, yr, ab, TOL)[0] == 0


@pytest.mark.parametrize("k", [8, 32])
def test_autotune_spmm(cuda, k):
    A = M.banded(50_000, 64, 24, seed=29)
    ents, best = autotune(A, k=k, reps=3)
    assert {e["format"] for e in ents} == {"csr", "sell"}
    assert all(e["opts"]["col_lanes"] * e["opts"]["cols_per_lane"] >= k
               for e in ents if e["format"] == "csr")
    # SELL: 4 (k <= 32) and 8 lanes per row, each with 32-bit / 16-bit columns
    sell = {(e["opts"]["lanes_per_row"], e["opts"]["index_mode"]) for e in ents
            if e["format"] == "sell"}
    assert sell == {(g, m) for g in (4, 8) for m in (_abi.INDEX_I32, _abi.INDEX_AUTO)}
    assert all(e["ms"] > 0 and e["status"] == 0 for e in ents)
    assert ents[best]["ms"] == min(e["ms"] for e in ents)


# ---- the batching configuration at full size ----------------------------------------------

def test_config4_banded_full(cuda):
    """1,048,576-row banded matrix (half-bandwidth 64, 24 per row), k = 1, 8, 32, row groups
    and SELL."""
    torch = cuda
    A = M.banded(1_048_576, 64, 24, seed=3)
    for k in (1, 8, 32):
        X, Xd = _x(torch, A.n, k, seed=30 + k)
        for fmt in ("csr", "sell"):
            Y = SpMatrix(A, fmt).spmm(Xd).cpu().numpy()
            for j in sorted({0, k // 2, k - 1}):
                yr, ab = O.csr_ref(A.rp, A.ci, A.v, np.ascontiguousarray(X[:, j]))
                assert O.rel_error(np.ascontiguousarray(Y[:, j]), yr, ab, TOL)[0] == 0


# ---- batches with k right-hand sides ------------------------------------------------------

def _batch_X(torch, b, k, seed, fp32=False):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    X = torch.rand((b.n, k), generator=g, dtype=torch.float64, device="cuda") * 2.0 - 1.0
    return X.float().double() if fp32 else X


def _check_batch_cols(mats, b, X, Y, tol, cols=None):
    """Every listed column of every matrix of the batch against the long-double product."""
    from pava_b200.batch_bench import union_csr
    U = union_csr(mats)
    for j in (range(X.shape[1]) if cols is None else cols):
        xj = X[:, j].contiguous().cpu().numpy().astype(np.float64)
        yr, ab = O.csr_ref(U.rp, U.ci, U.v, xj)
        yj = Y[:, j].contiguous().cpu().numpy()
        bad, mx, _ = O.rel_error(yj, yr, ab, tol)
        if bad:
            rows = np.abs(yj - yr) / np.maximum(np.maximum(np.abs(yr), ab), 1e-300) > tol
            which = sorted(set(np.searchsorted(b.y_offsets, np.nonzero(rows)[0], side="right") - 1))
            pytest.fail(f"column {j}: {bad} rows above {tol} (max {mx:.3e}), matrices {which[:8]}")


@pytest.mark.parametrize("k", [2, 8, 13, 32])
@pytest.mark.parametrize("fmt", ["csr", "sell", "auto"])
def test_batch_spmm_every_matrix_and_column(cuda, k, fmt):
    """k right-hand sides per matrix over the uneven batch (with an all-empty, a rectangular
    and a 1 x 1 matrix), one persistent launch, then the same launch captured and replayed."""
    torch = cuda
    mats = _batch_mats(60, seed=51)
    if fmt == "sell":  # the union's Poisson rows pad 1.85x: SELL takes it
        from pava_b200.batch_bench import union_csr
        assert M.sell_accepts(union_csr(mats))
    b = Batch(mats, fmt, k=k)
    if fmt == "auto":
        assert b.chosen()[0] in ("csr", "sell")
    X = _batch_X(torch, b, k, seed=52)
    Y = b.spmm(X)
    _check_batch_cols(mats, b, X, Y, TOL)
    Yg = torch.full_like(Y, float("nan"))
    b.capture_spmm(X, Yg)
    b.replay()
    torch.cuda.synchronize()
    assert torch.equal(Yg, Y), "graph replay differs from the direct launch"
    # strided X / Y (column slices of wider buffers)
    Xw = torch.zeros((b.n, k + 3), dtype=torch.float64, device="cuda")
    Xw[:, 1:k + 1] = X
    Yw = torch.full((b.m, k + 5), float("nan"), dtype=torch.float64, device="cuda")
    b.spmm(Xw[:, 1:k + 1], Yw[:, 2:k + 2])
    assert torch.equal(Yw[:, 2:k + 2], Y)
    assert torch.isnan(Yw[:, :2]).all() and torch.isnan(Yw[:, k + 2:]).all()


def test_batch_spmm_fp32c(cuda):
    torch = cuda
    mats = _batch_mats(30, seed=53)
    for A in mats:
        A.v = A.v.astype(np.float32).astype(np.float64)
    b = Batch(mats, "auto", precision=_abi.PREC_FP32C, k=8)
    X = _batch_X(torch, b, 8, seed=54, fp32=True)
    Y = b.spmm(X.float())
    _check_batch_cols(mats, b, X, Y, TOL32)


def test_batch_spmm_rejects_other_forms(cuda):
    mats = _batch_mats(4, seed=55)
    with pytest.raises(_abi.PavaError) as e:
        Batch(mats, "cvr", k=8)
    assert e.value.status == _abi.E_UNKNOWN_FORMAT
    b = Batch(mats, "csr5")
    torch = cuda
    X = torch.zeros((b.n, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(_abi.PavaError) as e:
        b.spmm(X)
    assert e.value.status == _abi.E_UNKNOWN_FORMAT


@pytest.mark.parametrize("k", [8, 32])
def test_config4_batch_4096_spmm_full_size(cuda, k):
    """The batching workload at full size with k right-hand sides: 4,096 matrices (rows
    log-uniform in [256, 32,768], Poisson(12) per row, 337 M nnz), autotuned for k, captured
    and replayed; every column of every matrix against the long-double product."""
    from pava_b200.batch_bench import batch_mats
    torch = cuda
    mats = batch_mats(4096)
    b = Batch(mats, "auto", k=k)
    X = _batch_X(torch, b, k, seed=60 + k)
    Y = torch.full((b.m, k), float("nan"), dtype=torch.float64, device="cuda")
    b.capture_spmm(X, Y)
    b.replay()
    torch.cuda.synchronize()
    _check_batch_cols(mats, b, X, Y, TOL)
    b.close()
