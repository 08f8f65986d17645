"""The learned selector on the GPU: device generators, feature extraction, the MLP's forward
and backward kernels against the CPU restatement (float64 numpy), training, selection, and
the regret on the committed training set against exhaustive autotuning."""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import selector_ref as R
from pava_b200 import _abi
from pava_b200 import matrices as M
from pava_b200 import selector as S
from pava_b200.api import SpMatrix

pytestmark = pytest.mark.gpu

DATA = os.path.join(os.path.dirname(__file__), "golden", "selector", "selector_timings.npz")


class _DevArray:
    """A device buffer seen through the CUDA array interface (no copy)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3}


def _host(A):
    """Device CSR -> numpy (rp, ci, v)."""
    import torch
    out = []
    for ptr, n, ts, dt in ((A.row_ptr, A.m + 1, "<i4", np.int32), (A.col_idx, A.nnz, "<i4", np.int32),
                           (A.vals, A.nnz, "<f8", np.float64)):
        if n == 0:
            out.append(np.empty(0, dt))
            continue
        out.append(torch.as_tensor(_DevArray(ptr, n, ts), device="cuda").cpu().numpy().copy())
    return tuple(out)


GEN = [
    ("stencil2d5", dict(family=_abi.GEN_STENCIL, m=4900, p0=2, p1=5, p2=0, p3=0)),
    ("stencil2d9", dict(family=_abi.GEN_STENCIL, m=5000, p0=2, p1=9, p2=0, p3=0)),
    ("stencil3d7", dict(family=_abi.GEN_STENCIL, m=8000, p0=3, p1=7, p2=0, p3=0)),
    ("stencil3d27", dict(family=_abi.GEN_STENCIL, m=9000, p0=3, p1=27, p2=0, p3=0)),
    ("banded", dict(family=_abi.GEN_BANDED, m=7000, p0=40, p1=17, p2=0, p3=0)),
    ("banded_wide", dict(family=_abi.GEN_BANDED, m=3000, p0=5, p1=30, p2=0, p3=0)),
    ("powerlaw", dict(family=_abi.GEN_POWERLAW, m=20000, p0=30.0, p1=1.5, p2=5000, p3=0.03)),
    ("blockdiag", dict(family=_abi.GEN_BLOCKDIAG, m=6000, p0=8, p1=64, p2=0, p3=0)),
]


@pytest.mark.parametrize("name,sp", GEN, ids=[g[0] for g in GEN])
def test_generator_valid_and_deterministic(cuda, name, sp):
    A = S.generate(sp, seed=5)
    B = S.generate(sp, seed=5)
    try:
        rp, ci, v = _host(A)
        rp2, ci2, v2 = _host(B)
        assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2) and np.array_equal(v, v2)
        assert rp[0] == 0 and rp[-1] == A.nnz and np.all(np.diff(rp) >= 0)
        assert ci.min() >= 0 and ci.max() < A.n
        L = np.diff(rp)
        rows = np.repeat(np.arange(A.m), L)
        inrow = np.ones(A.nnz, bool)
        inrow[rp[:-1][L > 0]] = False  # first element of each row
        assert np.all(np.diff(ci)[inrow[1:]] > 0), "columns not strictly increasing in a row"
        if sp["family"] == _abi.GEN_STENCIL:
            g = round(A.m ** (1 / sp["p0"]))
            assert g ** sp["p0"] == A.m
            if sp["p0"] == 2 and sp["p1"] == 5:
                assert A.nnz == 5 * g * g - 4 * g
            if sp["p0"] == 3 and sp["p1"] == 27:
                assert A.nnz == (3 * g - 2) ** 3
        if sp["family"] == _abi.GEN_BANDED:
            hb, k = int(sp["p0"]), int(sp["p1"])
            width = np.minimum(np.arange(A.m) + hb, A.n - 1) - np.maximum(np.arange(A.m) - hb, 0) + 1
            assert np.array_equal(L, np.minimum(k, width))
            assert np.all(np.abs(ci - rows) <= hb)
        if sp["family"] == _abi.GEN_BLOCKDIAG:
            assert L.min() >= 1 and L.max() <= 64
            # a dense block: every row's columns are consecutive and contain the row
            assert np.all(ci[rp[1:] - 1] - ci[rp[:-1]] + 1 == L)
            assert np.all((ci[rp[:-1]] <= np.arange(A.m)) & (np.arange(A.m) <= ci[rp[1:] - 1]))
        if sp["family"] == _abi.GEN_POWERLAW:
            assert abs((L == 0).mean() - sp["p3"]) < 0.01
            assert L.max() <= sp["p2"]
        assert abs(v.mean()) < 0.1 and abs(v.std() - 1) < 0.1
    finally:
        S.free(A)
        S.free(B)


@pytest.mark.parametrize("name,sp", GEN, ids=[g[0] for g in GEN])
def test_features_match_cpu(cuda, name, sp):
    A = S.generate(sp, seed=6)
    try:
        f = S.features(A)
        rp, ci, _ = _host(A)
        fr = R.features(rp, ci, A.n)
        assert np.allclose(f, fr, rtol=1e-5, atol=1e-5), (f, fr)
        assert np.array_equal(f, S.features(A))  # integer accumulation: same bits
    finally:
        S.free(A)


def test_features_host_matrices(cuda):
    import torch
    for A in (M.powerlaw(30_000, mean=12.0, p_empty=0.1, seed=7), M.laplace2d(100)):
        rp, ci = torch.from_numpy(A.rp).cuda(), torch.from_numpy(A.ci).cuda()
        csr = _abi.PavaCsr(A.m, A.n, A.nnz, rp.data_ptr(), ci.data_ptr(), 0, 1)
        f = np.zeros(12, np.float32)
        _abi.check(_abi.gpu().pava_features(ctypes.byref(csr), f.ctypes.data, None))
        assert np.allclose(f, R.features(A.rp, A.ci, A.n), rtol=1e-5, atol=1e-5)


def _random_problem(B, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(B, 12)).astype(np.float32)
    T = rng.normal(size=(B, R.OUT)).astype(np.float32)
    mask = (rng.uniform(size=(B, R.OUT)) > 0.1).astype(np.float32)
    return X, T, mask


def test_mlp_forward_matches_cpu(cuda):
    net = S.Network(seed=3)
    P, _, _ = net.params()
    X, _, _ = _random_problem(257, 8)
    Y = net.forward(X)
    Yr, _ = R.mlp_forward(P, X.astype(np.float64))
    assert np.allclose(Y, Yr, rtol=1e-4, atol=1e-4)


def test_mlp_gradient_matches_cpu(cuda):
    net = S.Network(seed=4)
    P, _, _ = net.params()
    X, T, mask = _random_problem(300, 9)
    net.set_batch(X, T, mask)
    loss, g = net.gradient()
    lr_, gr = R.mlp_loss_grad(P, X, T, mask)
    assert abs(loss - lr_) <= 1e-5 * max(1.0, abs(lr_))
    scale = np.abs(gr).max()
    assert np.max(np.abs(g - gr)) <= 1e-4 * scale, np.max(np.abs(g - gr)) / scale
    # the CPU restatement itself against central differences on a few parameters
    rng = np.random.default_rng(10)
    for p in rng.choice(R.NP, 12, replace=False):
        h = 1e-6
        Pp, Pm = P.astype(np.float64).copy(), P.astype(np.float64).copy()
        Pp[p] += h
        Pm[p] -= h
        fd = (R.mlp_loss_grad(Pp, X, T, mask)[0] - R.mlp_loss_grad(Pm, X, T, mask)[0]) / (2 * h)
        assert abs(fd - gr[p]) <= 1e-6 + 1e-4 * abs(gr[p])


def test_mlp_training_fits_a_teacher_and_is_deterministic(cuda):
    teacher = S.Network(seed=11)
    X, _, _ = _random_problem(1000, 12)
    T = teacher.forward(X)
    out = []
    for _ in range(2):
        net = S.Network(seed=13)
        net.set_batch(X, T)
        hist = net.train(1500, 3e-3)
        assert hist[-1] < 0.05 * hist[0], (hist[0], hist[-1])
        out.append(net.params()[0])
    assert np.array_equal(out[0], out[1])


def test_select_and_create_selected(cuda):
    import torch
    sp = dict(family=_abi.GEN_POWERLAW, m=200_000, p0=16.0, p1=1.5, p2=20_000, p3=0.02)
    A = S.generate(sp, seed=14)
    try:
        net = S.Network(seed=15)
        v, pred = net.select(A)
        assert 0 <= v < _abi.NVARIANTS and v == int(np.argmin(pred))
        rp, ci, vals = _host(A)
        x = M.uniform(A.n, seed=16)
        yr, ab = O.csr_ref(rp, ci, vals, x)
        for mlp in (net._h, None):  # the network, then the exhaustive fallback
            h = _abi.c_void_p()
            var = ctypes.c_int()
            _abi.check(_abi.gpu().pava_create_selected(ctypes.byref(A), mlp, None,
                                                       ctypes.byref(h), ctypes.byref(var)))
            xd = torch.from_numpy(x).cuda()
            y = torch.empty(A.m, dtype=torch.float64, device="cuda")
            _abi.check(_abi.gpu().pava_spmv(h, xd.data_ptr(), y.data_ptr(), None))
            torch.cuda.synchronize()
            _abi.gpu().pava_destroy(h)
            assert O.rel_error(y.cpu().numpy(), yr, ab, 1e-12)[0] == 0
            if mlp is not None:  # the network's pick, unless it is a SELL form that refuses A
                refused = S.FORM_FAMILY[v] == 6 and not M.sell_accepts(
                    M.from_arrays(A.m, A.n, rp, ci, vals))
                if refused:
                    order = [u for u in np.argsort(pred, kind="stable") if S.FORM_FAMILY[u] != 6]
                    assert var.value == order[0]
                else:
                    assert var.value == v
    finally:
        S.free(A)


def test_time_variants_all_run(cuda):
    sp = dict(family=_abi.GEN_BANDED, m=300_000, p0=64, p1=24, p2=0, p3=0)
    A = S.generate(sp, seed=17)
    try:
        ms, best = S.time_variants(A, reps=3)
        assert np.all(ms > 0) and best == int(np.argmin(ms))
    finally:
        S.free(A)


def test_selector_regret_on_training_set(cuda):
    """Trained on the committed timings of 2,000 matrices, evaluated on the 200 held-out ones:
    mean regret against the exhaustive autotune of all 32 forms <= 10 %, below the best single
    fixed form's and below choosing only the kernel variant (default tile parameters)."""
    assert os.path.exists(DATA), "tests/golden/selector/selector_timings.npz is missing"
    d = dict(np.load(DATA))
    assert int(d["n_train"]) == 2000 and int(d["n_test"]) == 200
    assert d["times_ms"].shape[1] == _abi.NVARIANTS
    _, rep = S.train_selector(d, epochs=3000, lr=3e-3, seed=0)
    assert rep["train_loss_last"] < 0.2 * rep["train_loss_first"]
    assert rep["selector_regret_mean"] <= 0.10, rep
    assert rep["selector_regret_mean"] < rep["fixed_regret_mean"], rep
    assert rep["selector_regret_mean"] < rep["variant_only_regret_mean"], rep


def test_selector_regret_on_fresh_timings(cuda):
    """Held out in time as well as in matrices: 24 matrices the training set never saw (seeds
    past its range, all four families), timed here on this GPU over all 32 forms (the full
    autotune); the network trained on the committed timings picks a form for each from its
    features alone (the smallest prediction among the forms that take the matrix, as
    pava_create_selected does).  Mean regret <= 10 %."""
    d = dict(np.load(DATA))
    net, _ = S.train_selector(d, epochs=3000, lr=3e-3, seed=0)
    regs, picks, bests = [], [], []
    for i in range(24):
        seed = 1_000_000 + i
        A = S.generate(S.spec(seed), seed=seed)
        try:
            ms, best = S.time_variants(A, reps=5)
            _, pred = net.select(A)
            v = int(S.choose(pred[None, :], ms[None, :])[0])
        finally:
            S.free(A)
        assert ms[best] > 0
        regs.append(ms[v] / ms[best] - 1.0 if ms[v] > 0 else np.inf)
        picks.append(v)
        bests.append(best)
    regs = np.array(regs)
    assert np.isfinite(regs).all(), (picks, bests)
    assert regs.mean() <= 0.10, (regs.round(3).tolist(), picks, bests)
