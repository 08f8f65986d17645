"""The floor kernels of the measurement library (include/pava_probe.h) compute what they claim:
their per-warp sums add up to the same totals as numpy over the same elements, and the TMA
gather4 path (mode 4) gathers exactly mode 1's values, with no bounded wait giving up."""
import numpy as np
import pytest

from pava_b200 import _abi
from pava_b200 import matrices as M

pytestmark = pytest.mark.gpu


def _floor(torch, P, mode, A, x, v, ci, bps=2):
    out = torch.empty(P.pava_probe_floor_out_len(bps, 256), dtype=torch.float64, device="cuda")
    assert P.pava_probe_floor(mode, v.data_ptr(), ci.data_ptr(), x.data_ptr(), A.nnz, A.n, 1,
                              bps, 256, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    return float(out.sum())


def test_floor_totals(cuda):
    torch = cuda
    P = _abi.probe()
    A = M.powerlaw(100_000, mean=12.0, seed=3)
    xh = M.uniform(A.n, seed=4)
    x, v, ci = (torch.from_numpy(a).cuda() for a in (xh, A.v, A.ci))
    ref = {0: float(np.sum(A.v * A.ci)), 2: float(np.sum(xh[A.ci])),
           3: float(np.sum(A.v * xh[A.ci]))}
    for mode, r in ref.items():
        got = _floor(torch, P, mode, A, x, v, ci)
        assert abs(got - r) <= 1e-9 * max(1.0, np.sum(np.abs(A.v) * np.abs(A.ci))), (mode, got, r)


@pytest.mark.parametrize("bps", [1, 4])
def test_tma_gather4_matches_load_unit_gathers(cuda, bps):
    torch = cuda
    P = _abi.probe()
    n, nnz = 1 << 20, 32 * 50_000
    xh = M.uniform(n, seed=5)
    x = torch.from_numpy(xh).cuda()
    ref = torch.empty(P.pava_probe_floor_out_len(2, 256), dtype=torch.float64, device="cuda")
    assert P.pava_probe_floor(1, 0, 0, x.data_ptr(), nnz, n, 1, 2, 256, ref.data_ptr(),
                              None) == 0
    out = torch.empty(P.pava_probe_floor_out_len(bps, 256), dtype=torch.float64, device="cuda")
    fail = torch.zeros(1, dtype=torch.int64, device="cuda")
    assert P.pava_probe_gather_tma(x.data_ptr(), nnz, n, 1, bps, out.data_ptr(),
                                   fail.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert int(fail.item()) == 0
    r, got = float(ref.sum()), float(out.sum())
    assert abs(got - r) <= 1e-9 * max(1.0, abs(r)), (got, r)
    # an odd n or a misaligned x is refused before any launch
    assert P.pava_probe_gather_tma(x.data_ptr(), nnz, n - 1, 1, bps, out.data_ptr(),
                                   fail.data_ptr(), None) == -10
    assert P.pava_probe_gather_tma(x.data_ptr() + 8, nnz, n - 2, 1, bps, out.data_ptr(),
                                   fail.data_ptr(), None) == -10
