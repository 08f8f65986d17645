"""Profiling driver: converts one benchmark matrix into one or more forms and runs a few SpMVs
of each, for ncu captures and for separating the cost of the x gathers from the streams.

    python -m pava_b200.profile_run --matrix c2 --variants cvr:steps=128 --reps 3
    python -m pava_b200.profile_run --matrix c3 \\
        --variants cvr:steps=64,csr5:sigma=16,cvr:steps=64;precision=1;index_mode=1

Matrices: c1 (512^2 Laplacian), c2 (power-law, 4,194,304 rows), c2local (c2's row lengths and
values with column j of row r replaced by min(r + j, n-1): the same streams, x gathers that hit
the same sectors), c3 (128^3 27-point stencil), banded (1,048,576 rows, half-bandwidth 64,
24 per row), batch (the block-diagonal union of ``--count`` of the batching workload's
matrices, values FP32-representable; 4,096 by default).  ``--rows`` shrinks c2 / banded for small captures.  A variant is
``format:key=value;...`` with the pava_opts keys (steps, sigma, tiles_per_chunk, precision
0=FP64 / 1=FP32C, index_mode 0=I32 / 1=DELTA16, lanes_per_row, col_lanes, cols_per_lane,
rows_per_tile, x_window).  ``--k K`` (CSR variants) times pava_spmm with K right-hand sides
instead of the SpMV.  Prints one JSON line per variant with the device time of the SpMV (or
SpMM) kernel (CUDA events) unless --quiet.

``--floor`` runs the floor kernels of include/pava_probe.h on the matrix's CSR arrays instead
(streams only, gathers at hashed columns only, column stream + gathers, values + columns +
gathers; mode 4: the gathers of mode 1 fetched by the TMA engine with tile::gather4, its total
checked against mode 1's), each over a sweep of blocks per SM, and prints the fastest launch
shape of each: the two costs an SpMV on this matrix is made of, measured apart.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def make_matrix(name, rows, count=4096):
    from . import matrices as M
    if name == "batch":
        from .batch_bench import batch_mats, union_csr
        return union_csr(batch_mats(count, fp32=True))
    if name == "c1":
        return M.laplace2d(512)
    if name == "c3":
        return M.stencil27(128)
    if name == "banded":
        return M.banded(rows if rows != 4_194_304 else 1_048_576, 64, 24)
    if name in ("c2", "c2local"):
        A = M.powerlaw(rows, seed=1)
        if name == "c2local":
            r = np.repeat(np.arange(A.m, dtype=np.int64), np.diff(A.rp))
            j = np.arange(A.nnz, dtype=np.int64) - np.repeat(A.rp[:-1].astype(np.int64), np.diff(A.rp))
            A.ci = np.minimum(r + j, A.n - 1).astype(np.int32)
        return A
    raise SystemExit(f"unknown matrix {name}")


def parse_variants(spec):
    out = []
    for item in spec.split(","):
        fmt, _, rest = item.partition(":")
        kw = {}
        for kv in filter(None, rest.split(";")):
            k, v = kv.split("=")
            kw[k] = int(v)
        out.append((fmt, kw))
    return out


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--matrix", default="c2")
    p.add_argument("--rows", type=int, default=4_194_304)
    p.add_argument("--variants", default="cvr:steps=128")
    p.add_argument("--reps", type=int, default=3)
    p.add_argument("--quiet", action="store_true")
    p.add_argument("--count", type=int, default=4096,
                   help="matrices in the batch union (--matrix batch)")
    p.add_argument("--k", type=int, default=1,
                   help="right-hand sides: k > 1 times pava_spmm on X (n x k, row-major); "
                        "CSR variants only")
    p.add_argument("--floor-modes", default="0,1,2,3",
                   help="floor kernels to run (0 streams, 1 gathers, 2 cols+gathers, 3 dot, "
                        "4 the gathers of 1 by TMA tile::gather4)")
    p.add_argument("--floor-bps", default="2,4,8,16", help="blocks per SM to sweep")
    p.add_argument("--floor", action="store_true",
                   help="time the floor kernels (pava_probe.h) on the matrix instead")
    p.add_argument("--flush", action="store_true",
                   help="write a 512 MB buffer between timed reps (matrices smaller than L2)")
    a = p.parse_args()

    import torch
    from . import _abi
    from .api import SpMatrix
    from . import matrices as M

    torch.cuda.set_device(0)
    _abi.check(_abi.gpu().pava_init(0))
    A = make_matrix(a.matrix, a.rows, a.count)
    x64 = M.uniform(A.n, seed=1, fp32=True)
    if a.floor:
        run_floors(torch, A, x64, max(a.reps, 1), a.quiet,
                   [int(t) for t in a.floor_modes.split(",")],
                   [int(t) for t in a.floor_bps.split(",")])
        return
    for fmt, kw in parse_variants(a.variants):
        prec = kw.get("precision", _abi.PREC_FP64)
        x = torch.from_numpy(x64).cuda()
        if prec == _abi.PREC_FP32C:
            x = x.float()
        try:
            mat = SpMatrix(A, fmt, **kw)
        except _abi.PavaError as e:
            print(json.dumps({"matrix": a.matrix, "format": fmt, "opts": kw, "error": str(e)}))
            continue
        y = torch.empty(A.m, dtype=torch.float64, device="cuda")
        if a.k > 1:
            X = torch.from_numpy(M.uniform(A.n * a.k, seed=2, fp32=True)).reshape(A.n, a.k)
            X = X.to("cuda", x.dtype)
            Y = torch.empty((A.m, a.k), dtype=torch.float64, device="cuda")
            try:  # a shape that cannot serve k is reported, not fatal
                mat.spmm(X, Y)
            except _abi.PavaError as e:
                print(json.dumps({"matrix": a.matrix, "format": fmt, "opts": kw, "k": a.k,
                                  "error": str(e)}))
                mat.close()
                continue
        s = torch.cuda.current_stream().cuda_stream
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(a.reps)]
        scratch = torch.empty(64 << 20, dtype=torch.float64, device="cuda") if a.flush else None
        for k in range(a.reps):
            if scratch is not None:
                scratch.fill_(float(k))  # evicts the matrix and x from the 126 MB L2
            ev[k][0].record()
            if a.k > 1:
                mat.spmm(X, Y)
            else:
                mat.spmv_raw(x.data_ptr(), y.data_ptr(), s, 1)
            ev[k][1].record()
            if a.k == 1:
                mat.spmv_raw(x.data_ptr(), y.data_ptr(), s, 2)
        torch.cuda.synchronize()
        if not a.quiet:
            info = mat.info()
            t = [e0.elapsed_time(e1) for e0, e1 in ev]
            best = min(t[1:]) if len(t) > 1 else t[0]
            print(json.dumps({"matrix": a.matrix, "format": fmt, "opts": kw, "m": A.m,
                              "nnz": A.nnz, "main_ms": t, "best_ms": best,
                              "k": a.k,
                              "alg_GBps": (info["alg_bytes"]
                                           + (a.k - 1) * (x.element_size() * A.n + 8.0 * A.m))
                              / (best * 1e-3) / 1e9,
                              "format_GBps": info["format_bytes"] / (best * 1e-3) / 1e9,
                              "alg_bytes": info["alg_bytes"],
                              "format_bytes": info["format_bytes"],
                              "convert_ms": info["convert_ms"]}), flush=True)
        mat.close()
        del mat


FLOOR_MODES = {0: ("streams", 12), 1: ("gathers", 0), 2: ("cols+gathers", 4),
               3: ("vals+cols+gathers", 12), 4: ("gathers by TMA gather4", 0)}


def run_floors(torch, A, x_host, reps, quiet, modes=(0, 1, 2, 3), bps_list=(2, 4, 8, 16)):
    """Floor kernels over A's nonzeros in CSR order: the best of blocks per SM in {2, 4, 8, 16}
    (256 threads) for each mode, CUDA-event timed, x resident in L2 as in an SpMV loop."""
    from . import _abi
    P = _abi.probe()
    ci = torch.from_numpy(A.ci).cuda()
    v = torch.from_numpy(A.v).cuda()
    x = torch.from_numpy(x_host).cuda()
    s = torch.cuda.current_stream().cuda_stream
    fail = torch.zeros(1, dtype=torch.int64, device="cuda")
    for mode in modes:
        name, bpe = FLOOR_MODES[mode]
        nnz = A.nnz if mode != 4 else A.nnz // 32 * 32  # whole warp steps for the TMA path
        best = None
        for bps in bps_list:
            out = torch.empty(P.pava_probe_floor_out_len(bps, 256), dtype=torch.float64,
                              device="cuda")
            if mode == 4:
                def launch(bps=bps, out=out):
                    return P.pava_probe_gather_tma(x.data_ptr(), nnz, A.n, 1, bps,
                                                   out.data_ptr(), fail.data_ptr(), s)
            else:
                def launch(bps=bps, out=out, mode=mode):
                    return P.pava_probe_floor(mode, v.data_ptr(), ci.data_ptr(), x.data_ptr(),
                                              A.nnz, A.n, 1, bps, 256, out.data_ptr(), s)
            for _ in range(2):
                if launch() != 0:
                    raise RuntimeError(f"floor mode {mode} failed")
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(reps)]
            for e0, e1 in ev:
                e0.record()
                launch()
                e1.record()
            torch.cuda.synchronize()
            t = sorted(e0.elapsed_time(e1) for e0, e1 in ev)[len(ev) // 2]
            if best is None or t < best[0]:
                best = (t, bps, float(out.sum()))
        t, bps, total = best
        line = {"floor": name, "mode": mode, "matrix_nnz": A.nnz, "n": A.n, "ms": t,
                "blocks_per_sm": bps, "threads": 256,
                "stream_GBps": bpe * A.nnz / (t * 1e-3) / 1e9 if bpe else None,
                "gathers_per_s": nnz / (t * 1e-3) if mode else None}
        if mode == 4:  # the same gathers as mode 1 over the same elements: the same total
            ref = torch.empty(P.pava_probe_floor_out_len(2, 256), dtype=torch.float64,
                              device="cuda")
            if P.pava_probe_floor(1, v.data_ptr(), ci.data_ptr(), x.data_ptr(), nnz, A.n, 1, 2,
                                  256, ref.data_ptr(), s) != 0:
                raise RuntimeError("floor mode 1 failed")
            r = float(ref.sum())
            line.update({"total": total, "mode1_total": r,
                         "totals_agree": abs(total - r) <= 1e-9 * max(1.0, abs(r)),
                         "wait_failures": int(fail.item())})
        if not quiet:
            print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
