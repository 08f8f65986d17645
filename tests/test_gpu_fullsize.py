"""Parity at full size on exactly the forms the benchmarks time.

* Power-law matrix (4,194,304 rows, ~66 M nnz, the headline workload): every FP64 candidate
  bench.py sweeps -- CVR steps 64 / 128, CSR5 sigma 16 / 32 -- against the long-double CSR
  product and against the reference's own first-call CVR and CSR5 output on the same inputs
  (cvr/cvr.h:2108 and csr5/csr5.h:149; the reference compiled from its sources where the CPU
  has AVX-512, else its bit-exact restatement).
* 128^3 27-point stencil (the precision workload): every form of bench.py's precision sweep,
  FP64 and FP32C with 16-bit column offsets, against the same three oracles.
* The 4,096-matrix batch (337 M nnz), FP64 and FP32C, autotuned, captured into a CUDA graph
  and replayed: every row of every matrix against the long-double CSR product.

Bounds: FP64 1e-12 relative per row, FP32C 1e-9 (cancellation-aware denominator
max(|y_ref_i|, sum_j |a_ij x_j|))."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from pava_b200 import _abi
from pava_b200 import matrices as M
from pava_b200.api import Batch, SpMatrix

pytestmark = pytest.mark.gpu

TOL = 1e-12
TOL32 = 1e-9
NCPU = os.cpu_count() or 1


def _reference_outputs(A, x):
    """The reference's first-call CVR and CSR5 results (y_cvr, y_csr5, which engine)."""
    if O.have_ref():
        y_cvr = O.ref_cvr(A.rp, A.ci, A.v, x, nthreads=NCPU)[0]
        y_csr5 = O.ref_csr5(A.rp, A.ci, A.v, x, nthreads=NCPU)[0]
        return y_cvr, y_csr5, "reference"
    y_cvr = O.cvr_port(A.rp, A.ci, A.v, x, nthreads=NCPU)[0]
    y_csr5 = O.csr5_port(A.rp, A.ci, A.v, x, nthreads=NCPU)[0]
    return y_cvr, y_csr5, "port"


def _gpu_y(torch, A, x, fmt, precision=_abi.PREC_FP64, **kw):
    mat = SpMatrix(A, fmt, precision=precision, **kw)
    dt = torch.float32 if precision == _abi.PREC_FP32C else torch.float64
    xd = torch.from_numpy(x).to("cuda", dt)
    y = torch.full((A.m,), float("nan"), dtype=torch.float64, device="cuda")
    mat.spmv(xd, y)
    y1 = y.cpu().numpy().copy()
    mat.spmv(xd, y)  # repeated calls give the same bits
    assert np.array_equal(y1, y.cpu().numpy())
    info = mat.info()
    mat.close()
    return y1, info


def _assert_all(y, oracles, ab, tol, what):
    for name, yo in oracles.items():
        bad, mx, mean = O.rel_error(y, yo, ab, tol)
        assert bad == 0, f"{what} vs {name}: {bad} rows above {tol}, max {mx:.3e}"


@pytest.fixture(scope="module")
def powerlaw_c2():
    A = M.powerlaw(4_194_304, seed=1)
    x = M.uniform(A.n, seed=1)
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    y_cvr, y_csr5, kind = _reference_outputs(A, x)
    return A, x, ab, {"csr_long_double": yr, f"{kind}_cvr": y_cvr, f"{kind}_csr5": y_csr5}


C2_FORMS = [("cvr", dict(steps=64)), ("cvr", dict(steps=128)), ("csr5", dict(sigma=16)),
            ("csr5", dict(sigma=32))]


@pytest.mark.parametrize("fmt,kw", C2_FORMS, ids=["cvr_steps64", "cvr_steps128",
                                                   "csr5_sigma16", "csr5_sigma32"])
def test_powerlaw_full_size_bench_forms(cuda, powerlaw_c2, fmt, kw):
    A, x, ab, oracles = powerlaw_c2
    assert A.m == 4_194_304 and A.nnz > 60_000_000
    y, info = _gpu_y(cuda, A, x, fmt, **kw)
    assert info["index_mode"] == _abi.INDEX_I32
    _assert_all(y, oracles, ab, TOL, f"{fmt} {kw}")


def test_powerlaw_full_size_sell_refused(cuda, powerlaw_c2):
    """Padding every 32-row slice of the lognormal rows to its longest row would store ~10x
    the nonzeros: the SELL form refuses the matrix instead of converting it."""
    A = powerlaw_c2[0]
    assert not M.sell_accepts(A) and M.sell_padded_elements(A) > 8 * A.nnz
    with pytest.raises(_abi.PavaError) as e:
        SpMatrix(A, "sell")
    assert e.value.status == _abi.E_UNSUPPORTED_PARAMS


@pytest.fixture(scope="module")
def stencil_c3():
    A = M.stencil27(128, seed=2)
    x = M.uniform(A.n, seed=3, fp32=True)
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    y_cvr, y_csr5, kind = _reference_outputs(A, x)
    return A, x, ab, {"csr_long_double": yr, f"{kind}_cvr": y_cvr, f"{kind}_csr5": y_csr5}


C3_FORMS = [("csr5", dict(sigma=32)), ("csr5", dict(sigma=32, tiles_per_chunk=8)),
            ("cvr", dict(steps=128)), ("sell", dict())]
C3_IDS = ["csr5_sigma32", "csr5_sigma32_tiles_per_chunk8", "cvr_steps128", "sell"]


@pytest.mark.parametrize("fmt,kw", C3_FORMS, ids=C3_IDS)
def test_stencil_full_size_fp64_forms(cuda, stencil_c3, fmt, kw):
    A, x, ab, oracles = stencil_c3
    assert A.nnz == 55_742_968
    y, _ = _gpu_y(cuda, A, x, fmt, **kw)
    _assert_all(y, oracles, ab, TOL, f"fp64 {fmt} {kw}")


@pytest.mark.parametrize("fmt,kw", C3_FORMS, ids=C3_IDS)
def test_stencil_full_size_fp32c_forms(cuda, stencil_c3, fmt, kw):
    """The FP32C forms bench.py's precision sweep times (16-bit column offsets); the fastest of
    them is the one the FP32C speed-up is quoted on."""
    A, x, ab, oracles = stencil_c3
    y, info = _gpu_y(cuda, A, x, fmt, precision=_abi.PREC_FP32C,
                     index_mode=_abi.INDEX_DELTA16, **kw)
    assert info["index_mode"] == _abi.INDEX_DELTA16
    _assert_all(y, oracles, ab, TOL32, f"fp32c {fmt} {kw}")
    # the compensated sums are far inside the bound on FP32-representable inputs
    assert O.rel_error(y, oracles["csr_long_double"], ab, 1e-12)[0] == 0


@pytest.mark.parametrize("precision", [_abi.PREC_FP64, _abi.PREC_FP32C], ids=["fp64", "fp32c"])
def test_batch_4096_full_size_graph_replay(cuda, precision):
    """The batching workload at full size: 4,096 matrices, rows log-uniform in [256, 32,768],
    Poisson(12) nonzeros per row, autotuned, run by graph replay; each matrix's rows against
    the long-double product of that matrix (the union is block diagonal, so one product over
    the union gives every matrix's own reference rows)."""
    from pava_b200.batch_bench import batch_mats, union_csr
    torch = cuda
    fp32 = precision == _abi.PREC_FP32C
    mats = batch_mats(4096, fp32=fp32)
    b = Batch(mats, "auto", precision=precision)
    assert b.count == 4096
    xs = [M.uniform(A.n, seed=7000 + i, fp32=fp32) for i, A in enumerate(mats)]
    xh = np.concatenate(xs)
    x = torch.from_numpy(xh).to("cuda", torch.float32 if fp32 else torch.float64)
    y = torch.full((b.m,), float("nan"), dtype=torch.float64, device="cuda")
    b.capture(x, y)
    b.replay()
    torch.cuda.synchronize()
    yg = y.cpu().numpy()
    y.fill_(float("nan"))
    b.replay()
    torch.cuda.synchronize()
    assert np.array_equal(y.cpu().numpy(), yg), "replays differ"
    U = union_csr(mats)
    yr, ab = O.csr_ref(U.rp, U.ci, U.v, xh)
    tol = TOL32 if fp32 else TOL
    bad, mx, _ = O.rel_error(yg, yr, ab, tol)
    if bad:
        rows = np.abs(yg - yr) / np.maximum(np.maximum(np.abs(yr), ab), 1e-300) > tol
        off = np.asarray(b.y_offsets)
        which = sorted(set(np.searchsorted(off, np.nonzero(rows)[0], side="right") - 1))
        pytest.fail(f"{bad} rows above {tol} (max {mx:.3e}) in matrices {which[:10]}")
    b.close()
