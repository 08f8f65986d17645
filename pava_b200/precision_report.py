"""FP32C error report: per matrix, the relative error per row of the FP32C forms (FP32 values
and x, FP64 y; CSR5 and CVR: compensated FP32 accumulation with FP64 carries; SELL, where it
takes the matrix: the exact products summed in FP64) against the FP64 form.

    python -m pava_b200.precision_report            # all matrices, full size
    python -m pava_b200.precision_report --only c3

Two errors per matrix and FP32C form, each as max and mean over rows of
|y - y_ref| / max(|y_ref|, sum_j |a_ij x_j|) (cancellation-aware denominator):

* arithmetic -- against the FP64 form run on the same FP32-rounded values and x: the error of
  the FP32C arithmetic alone (the bound the FP32C form is held to is 1e-9);
* total -- against the FP64 form on the original FP64 values and x: adds the rounding of the
  inputs to FP32 when they are not FP32-representable (about 1e-7 relative).

Matrices: c1 (512^2 5-point Laplacian, x ~ U[-1,1] FP64), c2 (4,194,304-row lognormal
power-law, values N(0,1) FP64), c3 (128^3 27-point stencil, values and x FP32-representable),
banded (1,048,576 rows, half-bandwidth 64, 24 per row, N(0,1)), batch (the 4,096-matrix
block-diagonal union, N(0,1)).  The FP64 reference is the library's FP64 drop-in, itself held
to 1e-12 of a long-double CSR product by the test suite.  One JSON line per matrix and form.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import _abi
from . import matrices as M
from .api import SpMatrix

FORMS32 = [("csr5", dict(sigma=32)), ("cvr", dict(steps=128)), ("sell", dict())]


def make(name):
    if name == "c1":
        return M.laplace2d(512), M.uniform(512 * 512, seed=0)
    if name == "c2":
        A = M.powerlaw(4_194_304, seed=1)
        return A, M.uniform(A.n, seed=1)
    if name == "c3":
        A = M.stencil27(128, seed=2)
        return A, M.uniform(A.n, seed=3, fp32=True)
    if name == "banded":
        A = M.banded(1_048_576, 64, 24, seed=3)
        return A, M.uniform(A.n, seed=61)
    if name == "batch":
        from .batch_bench import batch_mats, union_csr
        A = union_csr(batch_mats(4096))
        return A, M.uniform(A.n, seed=7)
    raise ValueError(name)


def rel(y, yref, absum):
    r = np.abs(y - yref) / np.maximum(np.maximum(np.abs(yref), absum), 1e-300)
    return float(r.max()), float(r.mean())


def absum_of(A, x):
    rows = np.repeat(np.arange(A.m, dtype=np.int64), np.diff(A.rp).astype(np.int64))
    return np.bincount(rows, weights=np.abs(A.v) * np.abs(x[A.ci]), minlength=A.m)


def report(torch, name):
    A, x = make(name)
    out = []
    xd = torch.from_numpy(x).cuda()
    y64 = SpMatrix(A, "csr5", sigma=32).spmv(xd).cpu().numpy()
    ab = absum_of(A, x)
    # the same matrix and x rounded to FP32, in FP64 arithmetic
    vr = A.v.astype(np.float32).astype(np.float64)
    xr = x.astype(np.float32).astype(np.float64)
    Ar = M.from_arrays(A.m, A.n, A.rp, A.ci, vr)
    y64r = SpMatrix(Ar, "csr5", sigma=32).spmv(torch.from_numpy(xr).cuda()).cpu().numpy()
    abr = absum_of(Ar, xr)
    x32 = xd.float()
    for fmt, kw in FORMS32:
        if fmt == "sell" and not M.sell_accepts(A):
            continue  # SELL refuses the matrix (padding)
        mat = SpMatrix(A, fmt, precision=_abi.PREC_FP32C, index_mode=_abi.INDEX_AUTO, **kw)
        y32 = mat.spmv(x32).cpu().numpy()
        im = mat.info()["index_mode"]
        mat.close()
        am, aa = rel(y32, y64r, abr)
        tm, ta = rel(y32, y64, ab)
        out.append({"matrix": name, "rows": A.m, "nnz": A.nnz,
                    "form": fmt + "".join(f"_{k}{v}" for k, v in kw.items()),
                    "columns": "16-bit" if im == _abi.INDEX_DELTA16 else "32-bit",
                    "inputs_fp32_representable": bool(np.array_equal(vr, A.v)
                                                      and np.array_equal(xr, x)),
                    "arithmetic_max": am, "arithmetic_mean": aa,
                    "total_max": tm, "total_mean": ta, "bound": 1e-9})
    return out


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--only", choices=["c1", "c2", "c3", "banded", "batch"], default=None)
    a = p.parse_args()
    import torch
    torch.cuda.set_device(0)
    _abi.check(_abi.gpu().pava_init(0))
    for name in ([a.only] if a.only else ["c1", "c2", "c3", "banded", "batch"]):
        for line in report(torch, name):
            print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
