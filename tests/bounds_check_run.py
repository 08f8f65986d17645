"""Runs the SpMV forms under the bounds-checked engine (libpava_gpu_bounds.so), in a process of
its own so that this library is the one ctypes loads; tests/test_gpu_bounds.py starts it.

    PAVA_GPU_LIB=pava_b200/lib/libpava_gpu_bounds.so python tests/bounds_check_run.py

Prints one JSON line: the largest relative error of the FP64 and the FP32C forms against the
long-double product (1e-12 / 1e-9 with no failed index test), and what the checks caught in a
CSR whose one column lies past n: the allocation-free entry point reads the caller's CSR
unvalidated, so a bad column reaches its kernel, which counts it and skips the element.  The
planted column is n + 3 and x is allocated with 64 spare entries, so even an unchecked read of
it would stay inside x's allocation."""
import ctypes
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    import numpy as np
    import torch

    from oracle import oracle as O
    from pava_b200 import _abi
    from pava_b200 import matrices as M
    from pava_b200.api import SpMatrix

    L = _abi.gpu()
    torch.cuda.set_device(0)
    _abi.check(L.pava_init(0))
    out = {"library": os.path.basename(_abi.gpu_lib_path()), "checked": L.pava_bounds_checked()}
    word = (ctypes.c_ulonglong * 3)()
    _abi.check(L.pava_bounds_report(word, 1))

    A = M.powerlaw(60_000, mean=16.0, cap=20_000, p_empty=0.05, seed=91)
    A32 = M.from_arrays(A.m, A.n, A.rp, A.ci, A.v.astype(np.float32).astype(np.float64))
    x = M.uniform(A.n, seed=92, fp32=True)
    yr, ab = O.csr_ref(A32.rp, A32.ci, A32.v, x)
    worst, worst32 = 0.0, 0.0
    forms = [("cvr", dict(steps=64)), ("cvr", dict(steps=128, index_mode=_abi.INDEX_AUTO)),
             ("csr5", dict(sigma=16)), ("csr5", dict(sigma=32, tiles_per_chunk=2)),
             ("csr", dict(lanes_per_row=8)),
             ("csr5", dict(sigma=32, precision=_abi.PREC_FP32C, index_mode=_abi.INDEX_AUTO)),
             ("cvr", dict(steps=64, precision=_abi.PREC_FP32C))]
    for fmt, kw in forms:
        mat = SpMatrix(A32, fmt, **kw)
        fp32 = kw.get("precision") == _abi.PREC_FP32C
        xd = torch.from_numpy(x).to("cuda", torch.float32 if fp32 else torch.float64)
        y = mat.spmv(xd).cpu().numpy()
        e = O.rel_error(y, yr, ab, 1e-9 if fp32 else 1e-12)[1]
        if fp32:
            worst32 = max(worst32, e)
        else:
            worst = max(worst, e)
        mat.close()
    # SELL (the power-law matrix pads too much for it) on a banded matrix and a stencil
    B = M.banded(20_000, 64, 24, seed=93)
    for S, kw in ((B, {}), (B, dict(precision=_abi.PREC_FP32C, index_mode=_abi.INDEX_AUTO)),
                  (M.stencil27(24, seed=96), dict(index_mode=_abi.INDEX_DELTA16))):
        S = M.from_arrays(S.m, S.n, S.rp, S.ci, S.v.astype(np.float32).astype(np.float64))
        xs_ = M.uniform(S.n, seed=97, fp32=True)
        fp32 = kw.get("precision") == _abi.PREC_FP32C
        mat = SpMatrix(S, "sell", **kw)
        xd = torch.from_numpy(xs_).to("cuda", torch.float32 if fp32 else torch.float64)
        y = mat.spmv(xd).cpu().numpy()
        ysr, absr = O.csr_ref(S.rp, S.ci, S.v, xs_)
        e = O.rel_error(y, ysr, absr, 1e-9 if fp32 else 1e-12)[1]
        if fp32:
            worst32 = max(worst32, e)
        else:
            worst = max(worst, e)
        mat.close()
    # multi-RHS through the X-window kernel
    X = M.uniform(B.n * 8, seed=94).reshape(B.n, 8)
    Y = SpMatrix(B, "csr", lanes_per_row=8, col_lanes=8, x_window=1).spmm(
        torch.from_numpy(X).cuda()).cpu().numpy()
    for j in range(8):
        yj, abj = O.csr_ref(B.rp, B.ci, B.v, np.ascontiguousarray(X[:, j]))
        worst = max(worst, O.rel_error(np.ascontiguousarray(Y[:, j]), yj, abj, 1e-12)[1])
    _abi.check(L.pava_bounds_report(word, 1))
    out.update({"max_rel_err_fp64": worst, "max_rel_err_fp32c": worst32,
                "failed_tests_clean": int(word[0])})

    # the planted column: the last element of the first non-empty row from row 7 on is n + 3
    ci = A.ci.copy()
    r = 7
    while A.rp[r + 1] == A.rp[r]:
        r += 1
    bad = int(A.rp[r + 1]) - 1
    ci[bad] = A.n + 3
    rp_d = torch.from_numpy(A.rp).cuda()
    ci_d = torch.from_numpy(ci).cuda()
    v_d = torch.from_numpy(A.v).cuda()
    xs = np.concatenate([M.uniform(A.n, seed=95), np.full(64, 1e300)])
    x_d = torch.from_numpy(xs).cuda()
    y_d = torch.empty(A.m, dtype=torch.float64, device="cuda")
    _abi.check(L.pava_spmv_csr_noalloc(A.m, A.n, A.nnz, rp_d.data_ptr(), ci_d.data_ptr(),
                                       v_d.data_ptr(), x_d.data_ptr(), y_d.data_ptr(), None))
    _abi.check(L.pava_bounds_report(word, 1))
    keep = np.ones(A.nnz, bool)
    keep[bad] = False
    rows = np.repeat(np.arange(A.m), np.diff(A.rp))
    y_expect = np.bincount(rows[keep], weights=A.v[keep] * xs[:A.n][A.ci[keep]], minlength=A.m)
    y = y_d.cpu().numpy()
    out.update({"planted_failed_tests": int(word[0]), "planted_site": int(word[1]),
                "planted_index": int(word[2]), "planted_n": A.n,
                "planted_row_skipped": bool(abs(y[r] - y_expect[r])
                                            <= 1e-12 * max(1.0, abs(y_expect[r]))),
                "planted_rows_finite": bool(np.isfinite(y).all())})
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
