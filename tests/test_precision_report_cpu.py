"""The error measures of the FP32C report (host side, no GPU)."""
import numpy as np

from pava_b200 import matrices as M
from pava_b200 import precision_report as P


def test_absum_matches_row_loop():
    A = M.powerlaw(2_000, mean=6.0, p_empty=0.1, seed=3)
    x = M.uniform(A.n, seed=4)
    ab = P.absum_of(A, x)
    for r in range(0, A.m, 97):
        s, e = A.rp[r], A.rp[r + 1]
        assert np.isclose(ab[r], np.sum(np.abs(A.v[s:e]) * np.abs(x[A.ci[s:e]])), rtol=1e-14)


def test_rel_uses_the_cancellation_aware_denominator():
    yref = np.array([1.0, 0.0, -2.0])
    y = np.array([1.0 + 1e-9, 1e-12, -2.0])
    ab = np.array([1.0, 1e-3, 4.0])
    mx, mean = P.rel(y, yref, ab)
    assert np.isclose(mx, 1e-9) and np.isclose(mean, (1e-9 + 1e-9) / 3)
