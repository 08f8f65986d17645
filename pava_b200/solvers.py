"""An iterative consumer of the engine: conjugate gradients on one converted matrix.

Every iteration calls the same handle's SpMV on device vectors, which is what exposes the
reference's repeated-call bug (its CVR and CSR5 kernels add into rows shared between threads
on each call, cvr/cvr.h:1415, csr5_spmv_avx512.h:277): here every call overwrites y, so the
iteration is correct however many times it runs.  With ``graph=True`` one iteration -- the
SpMV launches and the vector updates, scalars kept on the device -- is captured once into a
CUDA graph and replayed; the residual is read on the host only every ``check_every`` steps.

    x, info = cg(SpMatrix(A, "csr5"), b, tol=1e-10)
"""
from __future__ import annotations

import torch


def cg(mat, b, x0=None, tol: float = 1e-10, maxiter: int = 2000, check_every: int = 10,
       graph: bool = True):
    """Solves A x = b for a symmetric positive definite A held by ``mat`` (an FP64 SpMatrix of
    any form).  Stops when ||r|| <= tol * ||b|| (checked every ``check_every`` iterations).
    Returns (x, info) with info = {"iterations", "residual", "converged", "graph"}."""
    dev = b.device
    n = b.numel()
    x = torch.zeros(n, dtype=torch.float64, device=dev) if x0 is None else x0.clone()
    r = torch.empty_like(x)
    q = torch.empty_like(x)
    stream = torch.cuda.Stream(device=dev)
    stream.wait_stream(torch.cuda.current_stream(dev))

    def spmv(src, dst):
        mat.spmv_raw(src.data_ptr(), dst.data_ptr(), torch.cuda.current_stream(dev).cuda_stream, 0)

    with torch.cuda.stream(stream):
        spmv(x, q)
        r.copy_(b - q)
        p = r.clone()
        rr = torch.dot(r, r)
        bnorm = torch.linalg.vector_norm(b)

    def step():
        spmv(p, q)
        alpha = rr / torch.dot(p, q)
        x.add_(alpha * p)
        r.sub_(alpha * q)
        rr_new = torch.dot(r, r)
        p.mul_(rr_new / rr).add_(r)
        rr.copy_(rr_new)

    g = None
    if graph:
        with torch.cuda.stream(stream):
            step()  # warm-up outside the capture (allocator, kernels loaded)
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            step()
    it = 1 if graph else 0
    converged = False
    with torch.cuda.stream(stream):
        while it < maxiter:
            todo = min(check_every - it % check_every, maxiter - it)  # checks at multiples
            for _ in range(todo):
                if g is not None:
                    g.replay()
                else:
                    step()
            it += todo
            res = float(torch.sqrt(rr))
            if res <= tol * float(bnorm):
                converged = True
                break
    stream.synchronize()
    info = {"iterations": it, "residual": float(torch.sqrt(rr)) / float(bnorm),
            "converged": converged, "graph": g is not None}
    del g  # release the graph before its memory pool
    return x, info
