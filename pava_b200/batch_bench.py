"""Batching workloads: many uneven small matrices in one persistent launch replayed from a CUDA
graph, and a banded matrix with k right-hand sides; forms picked by the autotuner.

    python -m pava_b200.batch_bench                 # both workloads, full size
    python -m pava_b200.batch_bench --only banded --rows 262144
    python -m pava_b200.batch_bench --only batch --count 512

* batch:  4,096 square matrices, rows log-uniform in [256, 32,768], nnz per row Poisson(12),
  uniform distinct columns, values N(0,1); FP64 and FP32C (values rounded to FP32).  The
  union is autotuned (pava_autotune over its candidates, k = 1), converted into the winner,
  captured into a CUDA graph and replayed.
* banded: 1,048,576 rows, half-bandwidth 64, 24 distinct columns per row, X row-major n x k
  for k in {1, 8, 32}; the form is autotuned per k (k > 1: the CSR row-group shapes -- lanes
  per row, lanes across k, columns per lane, rows per tile -- and the SELL SpMM shapes).
* batch_spmm: the 4,096-matrix batch with k in {8, 32} right-hand sides per matrix, autotuned
  for k, one persistent launch captured into a CUDA graph and replayed.

Each line is one JSON object: device time per product (CUDA events, median of --reps after
warm-up; every input is larger than the 126 MB L2 except where noted), the compulsory
algorithmic bytes nnz*(s_v + s_i) + 4(m+1) + s_x*n*k + 8*m*k (s_i: 4 for 32-bit columns, 2 for
16-bit offsets), GB/s and the fraction of the
measured HBM copy bandwidth.  Parity with the oracle is the job of tests/test_gpu_batch.py;
here the graph replay is checked bit for bit against a direct launch, and the multi-RHS
product's first column against a single-vector product of the same form.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import _abi
from . import matrices as M
from .api import Batch, SpMatrix, autotune

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def time_it(torch, fn, reps, warmup=3):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts)), ts


def batch_mats(count, seed=41, lo=256, hi=32768, fp32=False):
    rng = np.random.default_rng(seed)
    mats = []
    for i in range(count):
        m = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        A = M.random_csr(m, mean=12.0, seed=seed * 100_000 + i)
        if fp32:
            A.v = A.v.astype(np.float32).astype(np.float64)
        mats.append(A)
    return mats


def union_csr(mats):
    """The block-diagonal union on the host (for the autotuner's table)."""
    rp = [np.zeros(1, np.int64)]
    ci, v = [], []
    r0 = c0 = z0 = 0
    for A in mats:
        rp.append(A.rp[1:].astype(np.int64) + z0)
        ci.append(A.ci.astype(np.int64) + c0)
        v.append(A.v)
        z0 += A.nnz
        c0 += A.n
        r0 += A.m
    return M.from_arrays(r0, c0, np.concatenate(rp), np.concatenate(ci), np.concatenate(v))


def run_batch(torch, count, reps, peak, precision):
    t0 = time.time()
    mats = batch_mats(count, fp32=precision == _abi.PREC_FP32C)
    gen_s = time.time() - t0
    t0 = time.time()
    b = Batch(mats, "auto", precision=precision)
    create_s = time.time() - t0
    # the autotuner's table for this union (the same search pava_batch_create ran)
    U = union_csr(mats)
    ents, best = autotune(U, k=1, precision=precision, reps=5)
    del U
    table = sorted(((e["format"], {k: v for k, v in e["opts"].items() if v and k != "precision"},
                     round(e["ms"], 4)) for e in ents if e["ms"] > 0), key=lambda t: t[2])
    fmt, opts = b.chosen()
    fp32 = precision == _abi.PREC_FP32C
    dt = torch.float32 if fp32 else torch.float64
    xs = [M.uniform(A.n, seed=7000 + i, fp32=fp32) for i, A in enumerate(mats)]
    x = torch.from_numpy(np.concatenate(xs)).to("cuda", dt)
    y = torch.empty(b.m, dtype=torch.float64, device="cuda")
    b.capture(x, y)
    ms, _ = time_it(torch, lambda: b.replay(), reps)
    yh = y.cpu().numpy()
    assert np.array_equal(yh, b.spmv(x).cpu().numpy()), "graph replay differs from a launch"
    sv = 4 if fp32 else 8
    si = 2 if b.info()["index_mode"] == _abi.INDEX_DELTA16 else 4  # column bytes as stored
    alg = b.nnz * (sv + si) + 4 * (b.m + count) + sv * b.n + 8 * b.m
    gbs = alg / (ms * 1e-3) / 1e9
    return {"workload": "batch", "matrices": count, "rows": b.m, "nnz": b.nnz,
            "precision": "fp32c" if fp32 else "fp64", "form": fmt,
            "opts": {k: v for k, v in opts.items() if v}, "index_bytes": si,
            "launch": "cuda graph replay",
            "ms": ms, "alg_bytes": alg, "GBps": gbs, "frac_hbm": gbs / peak[0],
            "peak": peak[1], "gen_s": gen_s,
            "create_s": create_s, "autotune": table}


def run_batch_spmm(torch, count, k, reps, peak):
    """The 4,096-matrix batch with k right-hand sides per matrix (X_i n_i x k, row-major,
    U[-1, 1]): autotuned for k, captured into a CUDA graph, replayed."""
    mats = batch_mats(count)
    t0 = time.time()
    b = Batch(mats, "auto", k=k)
    create_s = time.time() - t0
    fmt, opts = b.chosen()
    g = torch.Generator(device="cuda")
    g.manual_seed(100 + k)
    X = torch.rand((b.n, k), generator=g, dtype=torch.float64, device="cuda") * 2.0 - 1.0
    Y = torch.empty((b.m, k), dtype=torch.float64, device="cuda")
    b.capture_spmm(X, Y)
    ms, _ = time_it(torch, lambda: b.replay(), reps)
    Yr = Y.clone()
    b.spmm(X, Y)
    assert torch.equal(Y, Yr), "graph replay differs from a launch"
    alg = b.nnz * 12 + 4 * (b.m + count) + 8 * b.n * k + 8 * b.m * k
    gbs = alg / (ms * 1e-3) / 1e9
    return {"workload": "batch_spmm", "matrices": count, "rows": b.m, "nnz": b.nnz, "k": k,
            "precision": "fp64", "form": fmt, "opts": {kk: v for kk, v in opts.items() if v},
            "launch": "cuda graph replay (one persistent launch)", "ms": ms, "alg_bytes": alg,
            "GBps": gbs, "frac_hbm": gbs / peak[0], "peak": peak[1], "create_s": create_s}


def run_banded(torch, rows, ks, reps, peak):
    A = M.banded(rows, 64, 24, seed=3)
    out = []
    for k in ks:
        ents, best = autotune(A, k=k, reps=5)
        e = ents[best]
        opts = {kk: v for kk, v in e["opts"].items() if v and kk != "precision"}
        mat = SpMatrix(A, e["format"], **opts)
        X = M.uniform(A.n * k, seed=60 + k).reshape(A.n, k)
        Xd = torch.from_numpy(X).cuda()
        Y = torch.empty((A.m, k), dtype=torch.float64, device="cuda")
        if k > 1:  # a CSR row-group or a SELL SpMM shape
            ms, _ = time_it(torch, lambda: mat.spmm(Xd, Y), reps)
        else:
            ms, _ = time_it(torch, lambda: mat.spmv(Xd.reshape(-1), Y.reshape(-1)), reps)
        y0 = SpMatrix(A, "csr", lanes_per_row=8).spmv(Xd[:, 0].contiguous()).cpu().numpy()
        mx = float(np.max(np.abs(Y[:, 0].cpu().numpy() - y0)))
        si = 2 if mat.info()["index_mode"] == _abi.INDEX_DELTA16 else 4  # as stored
        alg = A.nnz * (8 + si) + 4 * (A.m + 1) + 8 * A.n * k + 8 * A.m * k
        gbs = alg / (ms * 1e-3) / 1e9
        ranked = sorted((x for x in ents if x["ms"] > 0), key=lambda x: x["ms"])
        out.append({"workload": "banded", "rows": A.m, "nnz": A.nnz, "k": k, "precision": "fp64",
                    "form": e["format"], "opts": opts, "index_bytes": si, "ms": ms,
                    "alg_bytes": alg, "GBps": gbs,
                    "frac_hbm": gbs / peak[0], "peak": peak[1], "max_abs_diff_vs_spmv_col0": mx,
                    "candidates": len(ents),
                    "runner_up_ms": ranked[1]["ms"] if len(ranked) > 1 else None,
                    "worst_ms": ranked[-1]["ms"]})
        mat.close()
    return out


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--only", choices=["batch", "banded", "batch_spmm"], default=None)
    p.add_argument("--count", type=int, default=4096)
    p.add_argument("--rows", type=int, default=1_048_576)
    p.add_argument("--reps", type=int, default=20)
    a = p.parse_args()
    import torch
    torch.cuda.set_device(0)
    _abi.check(_abi.gpu().pava_init(0))
    peak = hbm_peak()
    if a.only in (None, "banded"):
        for r in run_banded(torch, a.rows, (1, 8, 32), a.reps, peak):
            print(json.dumps(r), flush=True)
    if a.only in (None, "batch"):
        for prec in (_abi.PREC_FP64, _abi.PREC_FP32C):
            print(json.dumps(run_batch(torch, a.count, a.reps, peak, prec)), flush=True)
    if a.only in (None, "batch_spmm"):
        for k in (8, 32):
            print(json.dumps(run_batch_spmm(torch, a.count, k, a.reps, peak)), flush=True)


if __name__ == "__main__":
    main()
