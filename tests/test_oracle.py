"""The oracle pinned: its restatement of the reference CVR/CSR5 against the golden fixtures
(made by the reference itself, tests/golden/make_golden.py) and, on AVX-512 hosts, against the
reference compiled from its own sources (oracle/_ref)."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from pava_b200 import matrices as M

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _load(path):
    d = np.load(path)
    return {k: d[k] for k in d.files}


def test_golden_present():
    assert len(GOLDEN) >= 7


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_port_matches_golden(path):
    d = _load(path)
    T = int(d["threads"])
    y_cvr, _, _ = O.cvr_port(d["rp"], d["ci"], d["v"], d["x"], nthreads=T)
    y_csr5, _, _ = O.csr5_port(d["rp"], d["ci"], d["v"], d["x"], nthreads=T)
    # the restatement reproduces the reference bit for bit (same operation order)
    assert np.array_equal(y_cvr, d["y_cvr"])
    assert np.array_equal(y_csr5, d["y_csr5"])
    # and both agree with the long-double CSR product
    yr, ab = O.csr_ref(d["rp"], d["ci"], d["v"], d["x"])
    assert O.rel_error(y_cvr, yr, ab, 1e-13)[0] == 0
    assert O.rel_error(y_csr5, yr, ab, 1e-13)[0] == 0
    assert O.check_results(y_cvr, yr) == 0


def _rand(m, n, mean, seed, empty=0.02):
    A = M.powerlaw(m, n, mean=mean, cap=min(n, 4000), p_empty=empty, seed=seed)
    x = M.uniform(n, seed=seed + 1)
    return A, x


@pytest.mark.skipif(not O.have_ref(), reason="reference build needs AVX-512")
@pytest.mark.parametrize("T", [1, 3, 8])
@pytest.mark.parametrize("case", [(20000, 20000, 8.0, 1), (8000, 12000, 30.0, 2),
                                  (50000, 50000, 4.0, 3)])
def test_cvr_port_layout_bitexact_vs_reference(case, T):
    m, n, mean, seed = case
    A, x = _rand(m, n, mean, seed)
    y_ref, _, _, lay_ref = O.ref_cvr(A.rp, A.ci, A.v, x, nthreads=T, layout=True)
    lay = O.cvr_port_layout(A.rp, A.ci, A.v, T)
    for a, b in zip(lay_ref, lay):
        k = min(len(a), len(b))
        assert np.array_equal(a[:k], b[:k])
    y_port, _, _ = O.cvr_port(A.rp, A.ci, A.v, x, nthreads=T)
    assert np.array_equal(y_port, y_ref)


@pytest.mark.skipif(not O.have_ref(), reason="reference build needs AVX-512")
@pytest.mark.parametrize("T", [1, 4, 8])
@pytest.mark.parametrize("case", [(20000, 20000, 8.0, 4), (6000, 9000, 40.0, 5),
                                  (30000, 30000, 3.0, 6)])
def test_csr5_port_bitexact_vs_reference(case, T):
    m, n, mean, seed = case
    A, x = _rand(m, n, mean, seed, empty=0.05)
    y_ref, _, _, lay = O.ref_csr5(A.rp, A.ci, A.v, x, nthreads=T, layout=True)
    y_port, _, _ = O.csr5_port(A.rp, A.ci, A.v, x, nthreads=T)
    assert np.array_equal(y_port, y_ref)
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    assert O.rel_error(y_ref, yr, ab, 1e-13)[0] == 0


def test_rel_error_metric_flags_a_planted_mistake():
    A, x = _rand(3000, 3000, 10.0, 7)
    yr, ab = O.csr_ref(A.rp, A.ci, A.v, x)
    y, _, _ = O.cvr_port(A.rp, A.ci, A.v, x, nthreads=2)
    assert O.rel_error(y, yr, ab, 1e-12)[0] == 0
    y[17] += 1e-9 * max(abs(yr[17]), ab[17], 1.0)  # plant an error in the oracle's output
    bad, mx, _ = O.rel_error(y, yr, ab, 1e-12)
    assert bad == 1 and mx > 1e-12


def test_check_results_counts_one_percent_errors():
    y = np.array([1.0, 2.0, 3.0])
    assert O.check_results(y, y) == 0
    assert O.check_results(y * np.array([1.0, 1.02, 1.0]), y) == 1
