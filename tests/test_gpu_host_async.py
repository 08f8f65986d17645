"""The pipelined host-buffer entry point (pava_spmv_host_async): several calls in flight with
different inputs and outputs give, bit for bit, the device-buffer SpMV of each input."""
import numpy as np
import pytest

from pava_b200 import _abi
from pava_b200 import matrices as M
from pava_b200.api import SpMatrix

pytestmark = pytest.mark.gpu

FORMS = [("cvr", dict(steps=128)), ("csr5", dict(sigma=16)), ("csr", dict(lanes_per_row=8)),
         ("csr5", dict(sigma=32, precision=_abi.PREC_FP32C, index_mode=_abi.INDEX_DELTA16))]


@pytest.mark.parametrize("fmt,kw", FORMS, ids=["cvr", "csr5", "csr", "csr5_fp32c"])
def test_async_calls_match_device_spmv(cuda, fmt, kw):
    torch = cuda
    fp32 = kw.get("precision") == _abi.PREC_FP32C
    A = M.stencil27(40, seed=51) if fp32 else M.powerlaw(120_000, mean=16.0, cap=20_000, seed=52)
    mat = SpMatrix(A, fmt, **kw)
    dt = torch.float32 if fp32 else torch.float64
    xs = [torch.from_numpy(M.uniform(A.n, seed=60 + i, fp32=fp32)).to(dt).pin_memory()
          for i in range(5)]
    ys = [torch.full((A.m,), float("nan"), dtype=torch.float64).pin_memory() for _ in range(5)]
    stream = torch.cuda.Stream()
    for x, y in zip(xs, ys):
        mat.spmv_host_async(x, y, stream=stream)
    mat.wait()
    stream.synchronize()
    for x, y in zip(xs, ys):
        ref = mat.spmv(x.cuda()).cpu().numpy()
        assert np.array_equal(y.numpy(), ref)


def test_async_then_sync_entry_points_agree(cuda):
    torch = cuda
    A = M.laplace2d(200)
    mat = SpMatrix(A, "cvr")
    x = torch.from_numpy(M.uniform(A.n, seed=70)).pin_memory()
    y1 = torch.empty(A.m, dtype=torch.float64).pin_memory()
    mat.spmv_host_async(x, y1)
    torch.cuda.current_stream().synchronize()        # the caller's stream waits for the call
    y2 = mat.spmv_host(x.numpy())
    assert np.array_equal(y1.numpy(), y2)
