#!/usr/bin/env python
"""Headline benchmark: SpMV GB/s (% of HBM peak) on one B200 for the irregular power-law
matrix (4,194,304 x 4,194,304, lognormal rows with mean 16 and sigma 1.5, capped at 200,000,
2 % empty rows, ~64 M nnz, FP64 values N(0,1), x ~ U[-1,1], seed 1).

A step is one y = A x of the chosen variant (the fastest FP64 CVR / CSR5 form, picked by a
short timing sweep) with the matrix and x resident in HBM.  GB/s uses the compulsory byte
model nnz*(8+4) + 4(m+1) + 8n + 8m (x and y counted once).  The 852 MB a step streams is
larger than L2, so no flush is needed between steps; x (33.5 MB) stays L2-resident across
steps as it does in any SpMV loop.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pava|reference]

Under torchrun (N > 1) every rank runs its own replica (the path has no exchange step);
time is the max over ranks and value the aggregate of all ranks.  At N = 1 the line also
carries, measured after the timed region: `precision_form`, FP64 against the FP32C form on the
128^3 27-point stencil (speed-up and error; --no-precision skips it); `batch_form`, the
4,096-matrix batching workload (--no-batch); and `small_form`, the 512^2 Laplacian and the
banded matrix with L2 flushed before every SpMV (--no-small).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SpMV GB/s (% of HBM peak): chosen vs plain FP64 on B200 at stated rel. error"
WORKLOAD = ("irregular power-law FP64 SpMV: 4,194,304 x 4,194,304, lognormal row lengths "
            "(mean 16, sigma 1.5, cap 200,000, 2% empty rows), ~64M nnz, uniform distinct "
            "columns, values N(0,1), x ~ U[-1,1], seed 1")
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["pava", "reference"], default="pava")
    p.add_argument("--rows", type=int, default=4_194_304, help="smaller sizes for smoke runs")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-numa-local", dest="numa_local", action="store_false",
                   help="allocate the end-to-end run's pinned host buffers wherever the process "
                        "runs instead of on the GPU's NUMA node")
    p.add_argument("--no-batch", action="store_true",
                   help="skip the batching measurement (4,096-matrix union, k = 1 and 8)")
    p.add_argument("--no-precision", action="store_true",
                   help="skip the FP64 vs FP32C comparison on the 27-point stencil")
    p.add_argument("--no-small", action="store_true",
                   help="skip the 512^2 Laplacian / banded measurement")
    p.add_argument("--variants",
                   default="cvr:steps=64,cvr:steps=128,csr5:sigma=16,csr5:sigma=32,sell:",
                   help="FP64 candidates for the chosen variant")
    return p.parse_args()


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


def peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_from_profiles(kernel_key):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        for line in open(path):
            k, _, v = line.partition("=")
            if k.strip() == kernel_key:
                return float(v.split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thr = threading.Thread(target=self._read, daemon=True)
            self.thr.start()
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [t.strip() for t in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for nm, val in zip(names, f[3:7]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_local_cpus(index):
    """The CPUs of the NUMA node the GPU hangs off (sysfs local_cpulist of its PCI function),
    limited to those this process may use; None when unknown."""
    try:
        import torch
        p = torch.cuda.get_device_properties(index)
        path = (f"/sys/bus/pci/devices/{p.pci_domain_id:04x}:{p.pci_bus_id:02x}:"
                f"{p.pci_device_id:02x}.0/local_cpulist")
        cpus = set()
        for part in open(path).read().strip().split(","):
            if "-" in part:
                a, b = part.split("-")
                cpus |= set(range(int(a), int(b) + 1))
            elif part:
                cpus.add(int(part))
        cpus &= os.sched_getaffinity(0)
        return cpus or None
    except Exception:
        return None


def max_over_ranks(values, world, device):
    """Max over the ranks of each timing; every rank calls it with the same number of values,
    in the same order (a collective)."""
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(v) for v in t]


def aggregate_gbps(world, alg_bytes, ms):
    """Whole-job throughput of `world` replicas that each move alg_bytes per step in (at
    most) ms milliseconds."""
    return world * alg_bytes / (ms * 1e-3) / 1e9


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_cpu_bench(rows, iters, runs=3, formats="cvr,csr5"):
    """The reference's CPU CVR / CSR5 timed in a fresh process (oracle/cpu_bench.py): no CUDA
    context, no torch thread pools, OpenMP on every host core with OMP_PROC_BIND=close.
    Returns its JSON record."""
    env = dict(os.environ)
    for k in ("OMP_NUM_THREADS", "OMP_PROC_BIND", "OMP_PLACES"):
        env.pop(k, None)  # cpu_bench sets them for all host cores
    cmd = [sys.executable, "-m", "oracle.cpu_bench", "--rows", str(rows), "--iters", str(iters),
           "--runs", str(runs), "--formats", formats]
    out = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    if out.returncode != 0:
        raise RuntimeError(f"cpu_bench exited {out.returncode}: {out.stderr.strip()[-300:]}")
    return json.loads(out.stdout.strip().splitlines()[-1])


def cpu_record_summary(rec, best):
    r = rec["formats"][best]
    return (f"reference {best.upper()} on the full matrix ({rec['rows']:,} rows, {rec['nnz']:,} "
            f"nnz): one conversion ({r['convert_s']:.3f} s), then the median of {rec['runs']} runs "
            f"of {rec['iters']} timed SpMV calls ({r['s_per_spmv'] * 1e3:.3f} ms each), "
            f"{rec['cores']} OpenMP threads, OMP_PROC_BIND={rec['omp_proc_bind']}, "
            f"OMP_PLACES={rec['omp_places']}, {rec['cpu_model']}, in a process without CUDA")


def reference_arm(args, world, rank):
    """The reference's own CPU CVR and CSR5 (compiled from the reference's sources into
    oracle/_ref) on this box's host cores, on the same workload, metric and unit; the faster
    of the two is the line's value."""
    if rank != 0:
        return
    rec = run_cpu_bench(args.rows, iters=max(args.steps, 20))
    res = rec["formats"]
    best = max(res, key=lambda k: res[k]["GBps"])
    val, per = res[best]["GBps"], res[best]["s_per_spmv"]
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 3), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "rows": rec["rows"], "nnz": rec["nnz"], "chosen": best,
                   "l2": "inputs larger than L2"},
        "variants": {k: {"GB/s": round(v["GBps"], 3), "convert_s": v["convert_s"],
                         "s_per_spmv": v["s_per_spmv"]} for k, v in res.items()},
        "cpu_baseline": {"value": round(val, 3), "unit": "GB/s", "cores": rec["cores"],
                         "kind": rec["kind"], "cpu_model": rec["cpu_model"],
                         "sample": cpu_record_summary(rec, best)},
        "e2e": {"value": round(val, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        reference_arm(args, world, rank)
        return

    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    from pava_b200 import _abi
    from pava_b200 import matrices as M
    from pava_b200.api import SpMatrix

    _abi.check(_abi.gpu().pava_init(torch.cuda.current_device()))
    A = M.powerlaw(args.rows, seed=1)
    x_host = M.uniform(A.n, seed=1)
    alg = A.nnz * 12.0 + 4.0 * (A.m + 1) + 8.0 * A.n + 8.0 * A.m
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream
    x = torch.from_numpy(x_host).to(dev)
    y = torch.empty(A.m, dtype=torch.float64, device=dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def time_variant(mat, reps, stage=0):
        with torch.cuda.stream(stream):
            for _ in range(3):
                mat.spmv_raw(x.data_ptr(), y.data_ptr(), sp, stage)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(reps):
                mat.spmv_raw(x.data_ptr(), y.data_ptr(), sp, stage)
            b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / reps

    # candidates: FP64 CVR / CSR5 forms (the chosen one) and the plain FP64 CSR kernel
    variants = {}
    mats = {}
    refused = {}
    for fmt, kw in parse_variants(args.variants):
        name = fmt + "".join(f"_{k}{v}" for k, v in kw.items())
        try:
            mats[name] = SpMatrix(A, fmt, **kw)
        except _abi.PavaError as e:  # a form that does not take the matrix (SELL: padding)
            refused[name] = str(e)
            continue
        variants[name] = {"ms": time_variant(mats[name], 10),
                          "convert_ms": mats[name].info()["convert_ms"]}
    plain = SpMatrix(A, "csr")
    plain_ms = time_variant(plain, 10)
    chosen = min(variants, key=lambda k: variants[k]["ms"])
    for k in list(mats):
        if k != chosen:
            mats[k].close()
    mat = mats[chosen]
    info = mat.info()

    # timed region: K whole SpMVs (SpMV kernel + carry fixup, the fixup launched as a
    # programmatic dependent of the SpMV), then -- outside it -- K launches of the SpMV kernel
    # alone, each between two events, for the roofline of the dominant kernel
    K, W = args.steps, args.warmup
    with torch.cuda.stream(stream):
        for _ in range(W):
            mat.spmv_raw(x.data_ptr(), y.data_ptr(), sp, 0)
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clocks:
        barrier()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            start.record(stream)
            for k in range(K):
                mat.spmv_raw(x.data_ptr(), y.data_ptr(), sp, 0)
            stop.record(stream)
        stop.synchronize()
        torch.cuda.synchronize()
        barrier()
    ms = start.elapsed_time(stop) / K
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(K)]
    with torch.cuda.stream(stream):
        for k in range(K):
            ev[k][0].record(stream)
            mat.spmv_raw(x.data_ptr(), y.data_ptr(), sp, 1)
            ev[k][1].record(stream)
            mat.spmv_raw(x.data_ptr(), y.data_ptr(), sp, 2)
    torch.cuda.synchronize()
    main_ms = sum(a.elapsed_time(b) for a, b in ev) / K
    ms, main_ms = max_over_ranks([ms, main_ms], world, dev)

    # correctness of the timed variant (relative error against a long-double CSR product is
    # checked by the test suite; here the plain CSR kernel is the in-run check)
    # (cancellation-aware: |y - y_plain| / max(|y_plain|, sum_j |a_ij x_j|), the bound the
    # FP64 forms are held to, 1e-12)
    yc = y.cpu().numpy()
    yp = torch.empty_like(y)
    plain.spmv_raw(x.data_ptr(), yp.data_ptr(), None, 0)
    torch.cuda.synchronize()
    ypn = yp.cpu().numpy()
    rows = np.repeat(np.arange(A.m, dtype=np.int64), np.diff(A.rp))
    absum = np.bincount(rows, weights=np.abs(A.v) * np.abs(x_host[A.ci]), minlength=A.m)
    del rows
    den = np.maximum(np.maximum(np.abs(ypn), absum), 1e-300)
    max_rel_vs_plain = float(np.max(np.abs(yc - ypn) / den))

    # end-to-end through the public host-buffer entry point: every step copies x in from pinned
    # host memory, runs the SpMV and copies y out (pava_spmv_host_async: consecutive steps
    # overlap one step's copy-in, another's SpMV and a third's copy-out)
    # the pinned buffers on the GPU's own NUMA node (the copies then cross one socket link)
    saved = os.sched_getaffinity(0)
    local = gpu_local_cpus(torch.cuda.current_device()) if args.numa_local else None
    if local:
        os.sched_setaffinity(0, local)
    try:
        xh = torch.from_numpy(x_host).pin_memory()
        yh = torch.empty(A.m, dtype=torch.float64).pin_memory()
        yh.zero_()
    finally:
        if local:
            os.sched_setaffinity(0, saved)
    KE = max(3, K)
    for _ in range(2):
        mat.spmv_host_async(xh, yh, stream=stream)
    mat.wait()
    barrier()
    torch.cuda.synchronize()
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ea.record(stream)
    for _ in range(KE):
        mat.spmv_host_async(xh, yh, stream=stream)
    eb.record(stream)
    eb.synchronize()
    mat.wait()
    e2e_ms = ea.elapsed_time(eb) / KE
    e2e_ok = bool(np.array_equal(yh.numpy(), yc))
    e2e_ms, = max_over_ranks([e2e_ms], world, dev)

    peak, peak_kind = peak_hbm()
    achieved = alg / (main_ms * 1e-3) / 1e9
    kernel_key = f"{chosen}_main"
    traffic = traffic_from_profiles(kernel_key)
    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(args.rows)
        line = {
            "metric": METRIC,
            "value": round(aggregate_gbps(world, alg, ms), 3),
            "unit": "GB/s",
            "n_gpus": world,
            "steps": K,
            "warmup": W,
            "ms_per_step": round(ms, 6),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "rows": A.m, "nnz": A.nnz, "chosen": chosen,
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (852 MB streamed per step); x L2-resident",
                       "byte_model": "nnz*12 + 4(m+1) + 8n + 8m",
                       "alg_bytes_per_step": alg},
            "pct_of_hbm_peak": round(100.0 * alg / (ms * 1e-3) / 1e9 / peak, 2),
            "pct_of_8tbs_nominal": round(100.0 * alg / (ms * 1e-3) / 1e9 / 8000.0, 2),
            # the reference's CSR5 byte model (csr5/detail/utils.h getB: x counted per nonzero),
            # for comparison with the GB/s the reference prints
            "csr5_getB_GBps": round(((A.m + 1 + A.nnz) * 4.0 + (2.0 * A.nnz + A.m) * 8.0)
                                    / (ms * 1e-3) / 1e9, 3),
            "plain_fp64": {"format": "csr", "ms": round(plain_ms, 6),
                           "GB/s": round(alg / (plain_ms * 1e-3) / 1e9, 3)},
            "variants": {k: {"ms": round(v["ms"], 6), "GB/s": round(alg / (v["ms"] * 1e-3) / 1e9, 3),
                             "convert_ms": round(v["convert_ms"], 3)} for k, v in variants.items()},
            "variants_refused": refused,
            "max_rel_diff_vs_plain_csr": max_rel_vs_plain,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 3), "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "kernel": kernel_key, "kernel_ms": round(main_ms, 6)},
            "e2e": {"value": round(aggregate_gbps(world, alg, e2e_ms), 3), "unit": "GB/s",
                    "ms_per_step": round(e2e_ms, 6), "steps": KE, "h2d_bytes_per_step": 8 * A.n,
                    "d2h_bytes_per_step": 8 * A.m, "entry_point": "pava_spmv_host_async",
                    "y_equals_device_result": e2e_ok,
                    "pinned_on_gpu_numa_node": bool(local)},
            "gpu_launches": 2 * K,
            "clocks": clocks.summary(),
            "format_bytes_per_step": info["format_bytes"],
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if world == 1 and not args.no_precision:
            line["precision_form"] = precision_form(torch, stream)
        if world == 1 and not args.no_batch:
            line["batch_form"] = batch_form(torch)
        if world == 1 and not args.no_small:
            line["small_form"] = small_form(torch, stream, peak)
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def batch_form(torch, count=4096, reps=10):
    """The batching workload, measured after the timed region: 4,096 square matrices (rows
    log-uniform in [256, 32,768], Poisson(12) nonzeros per row, 337 M nnz, FP64), autotuned,
    captured into a CUDA graph and replayed -- one vector per matrix, and k = 8 right-hand sides
    per matrix (one persistent SpMM launch); median of `reps` replays, graph replay checked bit
    for bit against a direct launch.  GB/s by the compulsory bytes nnz*12 + 4(m + count) +
    8k(n + m)."""
    from pava_b200 import matrices as M
    from pava_b200.api import Batch
    from pava_b200.batch_bench import batch_mats
    try:
        mats = batch_mats(count)
        peak, _ = peak_hbm()
        out = {"workload": f"{count} matrices, rows log-uniform 256-32,768, Poisson(12) per row, "
                           "FP64, autotuned, CUDA graph replay"}
        for k in (1, 8):
            b = Batch(mats, "auto", k=k)
            fmt, opts = b.chosen()
            if k == 1:
                x = torch.from_numpy(np.concatenate(
                    [M.uniform(A.n, seed=7000 + i) for i, A in enumerate(mats)])).cuda()
                y = torch.empty(b.m, dtype=torch.float64, device="cuda")
                b.capture(x, y)
                direct = b.spmv(x).clone()
            else:
                g = torch.Generator(device="cuda")
                g.manual_seed(108)
                x = torch.rand((b.n, k), generator=g, dtype=torch.float64, device="cuda")
                y = torch.empty((b.m, k), dtype=torch.float64, device="cuda")
                b.capture_spmm(x, y)
                direct = b.spmm(x).clone()
            ts = []
            for _ in range(3):
                b.replay()
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                b.replay()
                e1.record()
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
            ms = float(np.median(ts))
            alg = b.nnz * 12.0 + 4.0 * (b.m + count) + 8.0 * k * (b.n + b.m)
            out[f"k{k}"] = {"form": fmt, "opts": {kk: v for kk, v in opts.items() if v},
                            "ms": round(ms, 4), "GB/s": round(alg / (ms * 1e-3) / 1e9, 1),
                            "frac_hbm": round(alg / (ms * 1e-3) / 1e9 / peak, 4),
                            "replay_equals_launch": bool(torch.equal(y, direct))}
            b.close()
        out.update({"rows": b.m, "nnz": b.nnz})
        return out
    except Exception as e:  # a side measurement; the headline line stands without it
        return {"unavailable": f"failed: {e}"}


def small_form(torch, stream, peak, reps=15):
    """FP64 SpMV on two more of the benchmark's matrices, each SpMV timed alone with L2 flushed
    first (a 256 MB write between reps; CUDA events on the stream, median of `reps` after 3
    warm-ups): the 512^2 5-point Laplacian (262,144 rows, 1,308,672 nnz, 21 MB: launch- and
    latency-bound) and the banded matrix (1,048,576 rows, half-bandwidth 64, 24 per row).
    Forms: CSR5 sigma 16, CVR steps 32, SELL with 32-bit columns and with 16-bit offsets; the
    fastest is reported with its GB/s (compulsory bytes, 12 per nonzero) and fraction of the
    copy bandwidth.  Then SpMM on the banded matrix with k = 8 and 32 right-hand sides (X and Y
    row-major, compulsory bytes 12 per nonzero + 8k per row of X and Y): the best row-group
    shape of the autotuner's earlier runs against the SELL SpMM."""
    from pava_b200 import _abi
    from pava_b200 import matrices as M
    from pava_b200.api import SpMatrix
    try:
        sp = stream.cuda_stream
        flush = torch.empty(32 << 20, dtype=torch.float64, device="cuda")
        out = {}
        for key, A in (("laplace512", M.laplace2d(512)), ("banded", M.banded(1_048_576, 64, 24))):
            x = torch.from_numpy(M.uniform(A.n, seed=5)).cuda()
            y = torch.empty(A.m, dtype=torch.float64, device="cuda")
            alg = A.nnz * 12.0 + 4.0 * (A.m + 1) + 8.0 * A.n + 8.0 * A.m
            forms = {}
            for fmt, kw in (("csr5", dict(sigma=16)), ("cvr", dict(steps=32)), ("sell", {}),
                            ("sell", dict(index_mode=_abi.INDEX_DELTA16))):
                mat = SpMatrix(A, fmt, **kw)
                ts = []
                with torch.cuda.stream(stream):
                    for r in range(reps + 3):
                        flush.fill_(float(r))
                        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        a.record(stream)
                        mat.spmv_raw(x.data_ptr(), y.data_ptr(), sp, 0)
                        b.record(stream)
                        b.synchronize()
                        if r >= 3:
                            ts.append(a.elapsed_time(b))
                mat.close()
                forms[fmt + "".join(f"_{k}{v}" for k, v in kw.items())] = float(np.median(ts))
            best = min(forms, key=forms.get)
            gbs = alg / (forms[best] * 1e-3) / 1e9
            out[key] = {"rows": A.m, "nnz": A.nnz, "form": best, "ms": round(forms[best], 5),
                        "GB/s": round(gbs, 1), "frac_hbm": round(gbs / peak, 4),
                        "forms_ms": {k: round(v, 5) for k, v in forms.items()}}
        # SpMM on the banded matrix: k = 8 and 32 right-hand sides, X and Y row-major, the best
        # row-group shape against the SELL SpMM
        A = M.banded(1_048_576, 64, 24)
        for k, shapes in ((8, (("csr", dict(lanes_per_row=4, col_lanes=4, cols_per_lane=2,
                                             rows_per_tile=32)),
                               ("sell", dict(lanes_per_row=4)))),
                          (32, (("csr", dict(lanes_per_row=8, col_lanes=8, cols_per_lane=4,
                                              rows_per_tile=16)),
                                ("sell", dict(lanes_per_row=8))))):
            X = torch.from_numpy(M.uniform(A.n * k, seed=6)).cuda().reshape(A.n, k)
            Y = torch.empty((A.m, k), dtype=torch.float64, device="cuda")
            alg = A.nnz * 12.0 + 4.0 * (A.m + 1) + 8.0 * k * (A.n + A.m)
            forms = {}
            for fmt, kw in shapes:
                mat = SpMatrix(A, fmt, **kw)
                ts = []
                with torch.cuda.stream(stream):
                    for r in range(reps + 3):
                        flush.fill_(float(r))
                        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        a.record(stream)
                        mat.spmm(X, Y, stream=stream)
                        b.record(stream)
                        b.synchronize()
                        if r >= 3:
                            ts.append(a.elapsed_time(b))
                mat.close()
                forms[fmt] = float(np.median(ts))
            best = min(forms, key=forms.get)
            gbs = alg / (forms[best] * 1e-3) / 1e9
            out[f"banded_spmm_k{k}"] = {"form": best, "ms": round(forms[best], 5),
                                        "GB/s": round(gbs, 1), "frac_hbm": round(gbs / peak, 4),
                                        "forms_ms": {f: round(v, 5) for f, v in forms.items()}}
        out["l2"] = "flushed before every SpMV / SpMM (256 MB write)"
        return out
    except Exception as e:  # a side measurement; the headline line stands without it
        return {"unavailable": f"failed: {e}"}


def precision_form(torch, stream):
    """The precision form on the 128^3 27-point stencil (2,097,152 rows, 55.7 M nnz, values and
    x FP32-representable): the fastest FP32C form (FP32 values and x, 16-bit column offsets)
    against the fastest FP64 form with 32-bit columns (the reference's 12 bytes per nonzero)
    and against the fastest FP64 form with 16-bit offsets, over the same small sweep (CSR5
    sigma 32 with 4 and 8 tiles per chunk; CVR steps 128; SELL), each timed as whole SpMVs
    (kernel + carry fixup) back to back, 30 after 5 warm-ups; the FP32C result's relative
    error per row against the FP64 result (cancellation-aware denominator)."""
    from pava_b200 import _abi
    from pava_b200 import matrices as M
    from pava_b200.api import SpMatrix
    try:
        A = M.stencil27(128, seed=2)
        xh = M.uniform(A.n, seed=3, fp32=True)
        sp = stream.cuda_stream
        x64 = torch.from_numpy(xh).cuda()
        x32 = x64.float()
        sweep = [("csr5", dict(sigma=32)), ("csr5", dict(sigma=32, tiles_per_chunk=8)),
                 ("cvr", dict(steps=128)), ("sell", dict())]
        out, ys = {}, {}
        for key, prec, x, extra in (
                ("fp64", _abi.PREC_FP64, x64, {}),
                ("fp64_d16", _abi.PREC_FP64, x64, dict(index_mode=_abi.INDEX_DELTA16)),
                ("fp32c", _abi.PREC_FP32C, x32, dict(index_mode=_abi.INDEX_DELTA16))):
            best = None
            for fmt, kw in sweep:
                mat = SpMatrix(A, fmt, precision=prec, **kw, **extra)
                y = torch.empty(A.m, dtype=torch.float64, device="cuda")
                with torch.cuda.stream(stream):
                    for _ in range(5):
                        mat.spmv_raw(x.data_ptr(), y.data_ptr(), sp, 0)
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    for _ in range(30):
                        mat.spmv_raw(x.data_ptr(), y.data_ptr(), sp, 0)
                    b.record(stream)
                b.synchronize()
                ms = a.elapsed_time(b) / 30
                name = fmt + "".join(f"_{k}{v}" for k, v in kw.items())
                out.setdefault("sweep_ms", {})[f"{key} {name}"] = round(ms, 6)
                if best is None or ms < best[1]:
                    best = (name, ms)
                    ys[key] = y.cpu().numpy()
                mat.close()
            out[key] = {"form": best[0], "ms": round(best[1], 6)}
        rows = np.repeat(np.arange(A.m, dtype=np.int64), np.diff(A.rp))
        absum = np.bincount(rows, weights=np.abs(A.v) * np.abs(xh[A.ci]), minlength=A.m)
        y64, y32 = ys["fp64"], ys["fp32c"]
        rel = np.abs(y32 - y64) / np.maximum(np.maximum(np.abs(y64), absum), 1e-300)
        out.update({"workload": "128^3 27-point stencil, 2,097,152 rows, "
                                f"{A.nnz:,} nnz, values and x FP32-representable",
                    "speedup_fp32c_over_fp64": round(out["fp64"]["ms"] / out["fp32c"]["ms"], 3),
                    "speedup_fp32c_over_fp64_d16": round(out["fp64_d16"]["ms"]
                                                         / out["fp32c"]["ms"], 3),
                    # against the reference's own format (CSR5, FP64, 32-bit columns)
                    "speedup_fp32c_over_fp64_csr5": round(
                        out["sweep_ms"]["fp64 csr5_sigma32"] / out["fp32c"]["ms"], 3),
                    "max_rel_err_vs_fp64": float(rel.max()),
                    "mean_rel_err_vs_fp64": float(rel.mean()), "error_bound": 1e-9})
        return out
    except Exception as e:  # a side measurement; the headline line stands without it
        return {"unavailable": f"failed: {e}"}


def cpu_baseline(rows):
    """The reference's CPU CVR and CSR5 (compiled from the reference's sources) on this box's
    host cores, on the full matrix, in a fresh process (the same measurement as the reference
    arm); the faster of the two."""
    try:
        rec = run_cpu_bench(rows, iters=100)
        res = rec["formats"]
        best = max(res, key=lambda k: res[k]["GBps"])
        return {"value": round(res[best]["GBps"], 3), "unit": "GB/s", "cores": rec["cores"],
                "kind": rec["kind"], "cpu_model": rec["cpu_model"],
                "sample": cpu_record_summary(rec, best),
                "variants": {k: round(v["GBps"], 3) for k, v in res.items()}}
    except Exception as e:  # the baseline is reported, never required
        return {"value": None, "unit": "GB/s", "cores": 0, "kind": "unavailable",
                "sample": f"failed: {e}"}


if __name__ == "__main__":
    main()
