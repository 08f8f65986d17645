"""ORACLE -- test and measurement infrastructure only: the CPU baseline.

Times the reference's own CPU CVR and CSR5 (oracle/_ref, compiled from the reference's sources;
the bit-exact C restatement where the CPU lacks AVX-512) on the power-law workload, in a
process of its own: no CUDA context and no torch thread pools share the host cores with it.

    python -m oracle.cpu_bench [--rows 4194304] [--iters 100] [--runs 3] [--formats cvr,csr5]

OpenMP runs on every host core this process may use (OMP_NUM_THREADS = that count,
OMP_PROC_BIND=close, OMP_PLACES=cores unless the caller set them), as the reference's
benchmark does (main.cpp:207 sets the thread count; run.sh pins with numactl).  Per format:
one conversion (timed, the reference's convertTime column), then `runs` runs of `iters` timed
SpMV calls after the checked first call (cvr/cvr.h:2108-2112, csr5/csr5.h:149-153); the median
run is reported.  Prints one JSON line: CPU model, cores, binding and per-format seconds per
SpMV and GB/s by the compulsory byte model nnz*12 + 4(m+1) + 8n + 8m.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def host_cpus():
    """Every CPU the machine has online, and the set this process may run on."""
    try:
        online = os.sched_getaffinity(0)
        allc = set(range(os.cpu_count() or 1))
        try:  # widen an affinity mask inherited from a parent that pinned itself
            os.sched_setaffinity(0, allc)
            online = os.sched_getaffinity(0)
        except OSError:
            pass
        return sorted(online)
    except AttributeError:
        return list(range(os.cpu_count() or 1))


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--rows", type=int, default=4_194_304)
    p.add_argument("--iters", type=int, default=100)
    p.add_argument("--runs", type=int, default=3)
    p.add_argument("--formats", default="cvr,csr5")
    a = p.parse_args(argv)
    cpus = host_cpus()
    # OpenMP reads these when the first parallel region starts (the libraries below are loaded
    # after this point)
    os.environ.setdefault("OMP_NUM_THREADS", str(len(cpus)))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from pava_b200 import matrices as M

    import numpy as np

    nthreads = int(os.environ["OMP_NUM_THREADS"])
    A = M.powerlaw(a.rows, seed=1)
    x = M.uniform(A.n, seed=1)
    alg = A.nnz * 12.0 + 4.0 * (A.m + 1) + 8.0 * A.n + 8.0 * A.m
    kind = "reference" if O.have_ref() else "port"
    res = {}
    for fmt in a.formats.split(","):
        if kind == "reference":
            f = O.ref_cvr if fmt == "cvr" else O.ref_csr5
        else:
            f = O.cvr_port if fmt == "cvr" else O.csr5_port
        runs, conv = [], None
        for _ in range(max(1, a.runs)):
            _, c, per = f(A.rp, A.ci, A.v, x, nthreads=nthreads, iters=max(1, a.iters))
            conv = c if conv is None else min(conv, c)
            runs.append(per)
        per = float(np.median(runs))
        res[fmt] = {"convert_s": conv, "s_per_spmv": per, "runs_s_per_spmv": runs,
                    "GBps": alg / per / 1e9}
    print(json.dumps({
        "kind": kind, "cpu_model": cpu_model(), "cores": nthreads, "cpus_online": len(cpus),
        "omp_proc_bind": os.environ.get("OMP_PROC_BIND"),
        "omp_places": os.environ.get("OMP_PLACES"), "rows": A.m, "nnz": A.nnz,
        "alg_bytes": alg, "iters": a.iters, "runs": a.runs, "formats": res}), flush=True)


if __name__ == "__main__":
    main()
