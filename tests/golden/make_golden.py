"""Generates the golden fixtures in tests/golden/ from the REFERENCE itself.

The reference's CVR and CSR5 engines are compiled from the reference tree into
oracle/_ref/libpava_ref.so (``make -C oracle ref``; needs an AVX-512 host) and run on small
seeded matrices from pava_b200.matrices.  For each case the fixture stores the CSR, x, and
the reference's first-call outputs: y of CVR (4 threads) and y of CSR5 (4 threads, sigma 12)
plus the CSR5 tile pointer and descriptor words, so the oracle's restatement can be pinned on
machines where the reference cannot run.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from pava_b200 import matrices as M  # noqa: E402

THREADS = 4


def cases():
    yield "laplace2d_g48", M.laplace2d(48), 0
    yield "powerlaw_m3000", M.powerlaw(3000, mean=16.0, cap=2000, seed=11), 1
    yield "powerlaw_m1500_longrows", M.powerlaw(1500, mean=24.0, sigma=2.0, cap=1500,
                                                p_empty=0.1, seed=12), 2
    yield "stencil27_g10", M.stencil27(10, seed=13), 3
    yield "banded_m1200", M.banded(1200, 64, 24, seed=14), 4
    yield "random_m2500_n3000", M.random_csr(2500, 3000, 12.0, seed=15), 5
    yield "blockdiag_m600", M.blockdiag(600, 8, 64, seed=16), 6


def main():
    O.build(ref=True)
    if not O.have_ref():
        raise SystemExit("the reference library needs an AVX-512 host")
    for name, A, seed in cases():
        x = M.uniform(A.n, -1.0, 1.0, seed=100 + seed)
        y_cvr, _, _ = O.ref_cvr(A.rp, A.ci, A.v, x, nthreads=THREADS)
        y_csr5, _, _, lay = O.ref_csr5(A.rp, A.ci, A.v, x, nthreads=THREADS, layout=True)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), m=A.m, n=A.n, rp=A.rp, ci=A.ci,
                            v=A.v, x=x, threads=THREADS, y_cvr=y_cvr, y_csr5=y_csr5,
                            csr5_tile_ptr=lay["tile_ptr"], csr5_tile_desc=lay["tile_desc"])
        print(name, A.m, A.nnz)


if __name__ == "__main__":
    main()
