"""Conjugate gradients over one converted matrix (pava_b200.solvers.cg): hundreds of SpMV
calls on the same handle, eager and replayed from a CUDA graph, converge to the known
solution -- which needs every call to overwrite y (the reference's kernels accumulate into
shared rows on repeated calls)."""
import numpy as np
import pytest

from oracle import oracle as O
from pava_b200 import matrices as M
from pava_b200.api import SpMatrix
from pava_b200.solvers import cg

pytestmark = pytest.mark.gpu

FORMS = [("cvr", dict(steps=64)), ("csr5", dict(sigma=16)), ("csr", dict(lanes_per_row=4))]


@pytest.mark.parametrize("fmt,kw", FORMS, ids=["cvr", "csr5", "csr"])
def test_cg_laplace(cuda, fmt, kw):
    torch = cuda
    A = M.laplace2d(128)                      # SPD, condition number ~ 6.6e3
    x_true = M.uniform(A.n, seed=41)
    b, _ = O.csr_ref(A.rp, A.ci, A.v, x_true)
    mat = SpMatrix(A, fmt, **kw)
    bd = torch.from_numpy(b).cuda()
    out = {}
    for graph in (False, True):
        x, info = cg(mat, bd, tol=1e-12, maxiter=3000, check_every=10, graph=graph)
        assert info["converged"], info
        xh = x.cpu().numpy()
        err = np.linalg.norm(xh - x_true) / np.linalg.norm(x_true)
        assert err < 1e-7, (err, info)
        out[graph] = (xh, info["iterations"])
    assert out[False][1] == out[True][1]
    assert np.allclose(out[False][0], out[True][0], rtol=1e-12, atol=1e-12)


def test_cg_residual_matches_oracle_product(cuda):
    """The residual the solver reports is the true one: recompute b - A x with the oracle."""
    torch = cuda
    A = M.laplace2d(96)
    b = M.uniform(A.n, seed=42)
    x, info = cg(SpMatrix(A, "cvr", steps=128), torch.from_numpy(b).cuda(), tol=1e-11)
    ax, _ = O.csr_ref(A.rp, A.ci, A.v, x.cpu().numpy())
    res = np.linalg.norm(b - ax) / np.linalg.norm(b)
    assert info["converged"] and res < 1e-10, (res, info)
