"""The learned form selector: training set generation, GPU training, selection and regret.

    python -m pava_b200.selector generate --out tests/golden/selector/selector_timings.npz
    python -m pava_b200.selector evaluate --data tests/golden/selector/selector_timings.npz

Training set: 2,000 training and 200 held-out matrices; matrix i is drawn from a generator
seeded with i.  Families (in turn): stencil (2-D 5/9-point, 3-D 7/27-point), banded-random,
lognormal power-law and block-diagonal (dense blocks of 8..64); rows log-uniform in
[10^4, 10^7] and nonzeros log-uniform in [10^5, 10^8] (each family's row length follows
from the pair, within its own range); values N(0,1), FP64.  Every matrix is generated on the
GPU (pava_gen_device), described by its 12 structural features (pava_features), and each of
the 32 engine forms -- seven kernel variants with their tile parameters, the k = 1 candidate
set of pava_autotune -- is converted and timed on it (pava_time_variants: median of 5
CUDA-event timings after two warm-ups, x and y resident).  The file keeps the features, the
times and each matrix's family, rows and nonzeros.

Network: MLP 12-64-64-32 (ReLU, FP32), trained on the GPU by the library's own kernels
(pava_mlp_train: full-batch Adam on the masked mean squared error of standardised
log-times).  Selection = the form with the smallest predicted log-time among the forms that
take the matrix (a SELL form refuses a matrix whose slice padding would more than double it,
and pava_create_selected then moves to the next prediction); a kernel variant's predicted
time is the smallest over its forms.  Regret of a choice = t_chosen / t_best - 1, t_best
from the exhaustive timing of all 32 forms (the full autotune).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time

import numpy as np

from . import _abi

FAMILIES = ["stencil", "banded", "powerlaw", "blockdiag"]
FAMILY_NAMES = ["cvr_s64", "cvr_s128", "csr5_s16", "csr5_s32", "csr_l1_4", "csr_l8_32", "sell"]


def _form_names():
    out = []
    for s_ in (64, 128):
        for a in ("i32", "auto"):
            out.append(f"cvr_s{s_}_{a}")
    for sg in (16, 32):
        for w in ("tiles_default", "tiles_wave"):
            for a in ("i32", "auto"):
                out.append(f"csr5_s{sg}_{w}_{a}")
    for gl in (1, 2, 4, 8, 16, 32):
        for g in (1, 4, 16):
            out.append(f"csr_l{gl}_g{g}")
    out += ["sell_i32", "sell_auto"]
    return out


FORM_NAMES = _form_names()
# the kernel variant each form belongs to (pava_variant_family)
FORM_FAMILY = np.array([0, 0, 1, 1] + [2] * 4 + [3] * 4 + [4] * 9 + [5] * 9 + [6] * 2)
# each variant's default form, the one a selector of the kernel variant alone would run (CVR /
# CSR5 / SELL with default tiles and 32-bit columns, CSR 4 and 32 lanes with 4 row groups per
# tile)
FAMILY_DEFAULT_FORM = np.array([0, 2, 4, 8, 12 + 3 * 2 + 1, 12 + 3 * 5 + 1, 30])
N_TRAIN, N_TEST = 2000, 200


# ---- training-set matrices ----------------------------------------------------------------

def spec(i: int) -> dict:
    """Generator parameters of matrix i (seeded with i)."""
    rng = np.random.default_rng(i)
    fam = FAMILIES[i % 4]
    rows = float(np.exp(rng.uniform(np.log(1e4), np.log(1e7))))
    nnz = float(np.exp(rng.uniform(np.log(1e5), np.log(1e8))))

    def fit_rows(per_row):  # rows in [1e4, 1e7] with rows * per_row in [1e5, 1e8]
        lo = max(1e4, 1e5 / per_row)
        hi = min(1e7, 1e8 / per_row)
        return int(min(max(rows, lo), hi)) if lo <= hi else int(lo)

    if fam == "stencil":
        kinds = [(2, 5), (3, 7), (2, 9), (3, 27)]
        want = nnz / rows
        dims, pts = min(kinds, key=lambda k: abs(np.log(k[1]) - np.log(max(want, 1.0))))
        # a g^dims grid with g^dims in [1e4, 1e7] (the generator keeps g^dims <= m)
        g = int(np.ceil(fit_rows(pts) ** (1.0 / dims) - 1e-9))
        while g ** dims > 1e7:
            g -= 1
        while g ** dims < 1e4:
            g += 1
        return dict(family=_abi.GEN_STENCIL, m=g ** dims, p0=dims, p1=pts, p2=0, p3=0,
                    name=f"stencil{dims}d{pts}")
    if fam == "banded":
        per_row = int(np.clip(round(nnz / rows), 2, 512))
        hb = int(max(per_row, round(per_row * rng.uniform(0.5, 8.0))))
        return dict(family=_abi.GEN_BANDED, m=fit_rows(per_row), p0=hb, p1=per_row, p2=0, p3=0,
                    name="banded")
    if fam == "powerlaw":
        mean = float(np.clip(nnz / rows, 2.0, 1000.0))
        sigma = float(rng.uniform(0.5, 2.0))
        m = fit_rows(mean)
        return dict(family=_abi.GEN_POWERLAW, m=m, p0=mean, p1=sigma, p2=min(200_000, m),
                    p3=float(rng.uniform(0.0, 0.05)), name="powerlaw")
    return dict(family=_abi.GEN_BLOCKDIAG, m=fit_rows(42.0), p0=8, p1=64, p2=0, p3=0,
                name="blockdiag")


def generate(sp: dict, seed: int) -> _abi.PavaCsr:
    """Builds the matrix on the device (free it with free())."""
    q = _abi.PavaGenParams(sp["family"], sp["m"], 0, sp["p0"], sp["p1"], sp["p2"], sp["p3"])
    A = _abi.PavaCsr()
    _abi.check(_abi.gpu().pava_gen_device(ctypes.byref(q), seed, None, ctypes.byref(A)))
    return A


def free(A: _abi.PavaCsr) -> None:
    _abi.gpu().pava_free_device_csr(ctypes.byref(A))


def features(A: _abi.PavaCsr) -> np.ndarray:
    f = np.zeros(_abi.MLP_IN, np.float32)
    _abi.check(_abi.gpu().pava_features(ctypes.byref(A), f.ctypes.data, None))
    return f


def time_variants(A: _abi.PavaCsr, reps: int = 5):
    ms = np.zeros(_abi.NVARIANTS, np.float64)
    best = ctypes.c_int()
    _abi.check(_abi.gpu().pava_time_variants(ctypes.byref(A), reps, ms.ctypes.data,
                                             ctypes.byref(best)))
    return ms, best.value


def build_dataset(n_train=N_TRAIN, n_test=N_TEST, reps=5, log_every=100):
    total = n_train + n_test
    F = np.zeros((total, _abi.MLP_IN), np.float32)
    T = np.zeros((total, _abi.NVARIANTS), np.float64)
    fam = np.zeros(total, np.int32)
    rows = np.zeros(total, np.int64)
    nnz = np.zeros(total, np.int64)
    t0 = time.time()
    for i in range(total):
        sp = spec(i)
        A = generate(sp, seed=i)
        try:
            F[i] = features(A)
            T[i], _ = time_variants(A, reps)
            fam[i], rows[i], nnz[i] = sp["family"], A.m, A.nnz
        finally:
            free(A)
        if log_every and (i + 1) % log_every == 0:
            print(f"  {i + 1}/{total} matrices, {time.time() - t0:.1f} s", flush=True)
    return dict(features=F, times_ms=T, family=fam, rows=rows, nnz=nnz,
                n_train=np.int64(n_train), n_test=np.int64(n_test), reps=np.int64(reps))


# ---- network ------------------------------------------------------------------------------

class Network:
    """pava_mlp: the MLP 12-64-64-32 living on the GPU."""

    def __init__(self, seed: int = 0):
        h = _abi.c_void_p()
        _abi.check(_abi.gpu().pava_mlp_create(seed, ctypes.byref(h)))
        self._h = h

    def set_norm(self, mean, std):
        mean = np.ascontiguousarray(mean, np.float32)
        std = np.ascontiguousarray(std, np.float32)
        _abi.check(_abi.gpu().pava_mlp_set_params(self._h, None, mean.ctypes.data, std.ctypes.data))

    def params(self):
        P = np.zeros(_abi.MLP_NPARAM, np.float32)
        mu = np.zeros(_abi.MLP_IN, np.float32)
        sd = np.zeros(_abi.MLP_IN, np.float32)
        _abi.check(_abi.gpu().pava_mlp_get_params(self._h, P.ctypes.data, mu.ctypes.data,
                                                  sd.ctypes.data))
        return P, mu, sd

    def set_params(self, P):
        P = np.ascontiguousarray(P, np.float32)
        _abi.check(_abi.gpu().pava_mlp_set_params(self._h, P.ctypes.data, None, None))

    def set_batch(self, X, T=None, mask=None):
        X = np.ascontiguousarray(X, np.float32)
        Tp = None if T is None else np.ascontiguousarray(T, np.float32)
        Mp = None if mask is None else np.ascontiguousarray(mask, np.float32)
        self._batch = (X, Tp, Mp)
        _abi.check(_abi.gpu().pava_mlp_set_batch(self._h, X.shape[0], X.ctypes.data,
                                                 None if Tp is None else Tp.ctypes.data,
                                                 None if Mp is None else Mp.ctypes.data))

    def forward(self, X):
        self.set_batch(X)
        Y = np.zeros((len(X), _abi.MLP_OUT), np.float32)
        _abi.check(_abi.gpu().pava_mlp_forward(self._h, Y.ctypes.data))
        return Y

    def gradient(self):
        g = np.zeros(_abi.MLP_NPARAM, np.float32)
        loss = ctypes.c_float()
        _abi.check(_abi.gpu().pava_mlp_gradient(self._h, g.ctypes.data, ctypes.byref(loss)))
        return loss.value, g

    def train(self, epochs: int, lr: float):
        hist = np.zeros(epochs, np.float32)
        _abi.check(_abi.gpu().pava_mlp_train(self._h, epochs, lr, hist.ctypes.data))
        return hist

    def select(self, A: _abi.PavaCsr):
        v = ctypes.c_int()
        pred = np.zeros(_abi.MLP_OUT, np.float32)
        _abi.check(_abi.gpu().pava_select(self._h, ctypes.byref(A), ctypes.byref(v),
                                          pred.ctypes.data))
        return v.value, pred

    def close(self):
        if getattr(self, "_h", None):
            _abi.gpu().pava_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def targets(times_ms):
    """log-times, masked where a variant failed (time < 0)."""
    mask = (times_ms > 0).astype(np.float32)
    logt = np.log(np.where(times_ms > 0, times_ms, 1.0))
    return logt, mask


def regret(times_ms, choice):
    t = np.where(times_ms > 0, times_ms, np.inf)
    best = t.min(axis=1)
    chosen = t[np.arange(len(t)), choice]
    return chosen / best - 1.0


def choose(pred, times_ms):
    """The selection rule of pava_create_selected: the smallest prediction among the forms that
    take the matrix (a form that refused it has no time; its refusal costs one conversion
    attempt, which regret does not count)."""
    return np.where(times_ms > 0, pred, np.inf).argmin(1)


def train_selector(data, epochs=3000, lr=3e-3, seed=0):
    """Trains on the first n_train matrices; returns the network and a report on the held-out
    ones (selector regret, the regret of the best single fixed variant, and of a row-length
    rule), all against exhaustive timing."""
    F, Tms = data["features"], data["times_ms"]
    ntr = int(data["n_train"])
    Ftr, Fte = F[:ntr], F[ntr:]
    logt, mask = targets(Tms)
    mu_f = Ftr.mean(0)
    sd_f = Ftr.std(0)
    sd_f = np.where(sd_f > 1e-6, sd_f, 1.0)
    mt = logt[:ntr][mask[:ntr] > 0]
    mu_t, sd_t = float(mt.mean()), float(mt.std() or 1.0)
    T = ((logt - mu_t) / sd_t).astype(np.float32)
    net = Network(seed)
    net.set_norm(mu_f, sd_f)
    net.set_batch(Ftr, T[:ntr], mask[:ntr])
    hist = net.train(epochs, lr)
    pred_tr = net.forward(Ftr)
    pred = net.forward(Fte)
    choice = choose(pred, Tms[ntr:])
    reg = regret(Tms[ntr:], choice)
    # without the network: the one variant that is best on average over the training set
    tr_reg = np.stack([regret(Tms[:ntr], np.full(ntr, v)) for v in range(_abi.NVARIANTS)])
    fixed = int(np.argmin(np.where(np.isfinite(tr_reg), tr_reg, 1e9).mean(1)))
    reg_fixed = regret(Tms[ntr:], np.full(len(Fte), fixed))
    # the network asked only for the kernel variant, each variant run with its default tile
    # parameters: what predicting the tile parameters adds
    fam_pred = np.stack([np.where(FORM_FAMILY == f, pred, np.inf).min(1)
                         for f in range(_abi.NFAMILIES)], 1)
    fam_pred = np.where(Tms[ntr:][:, FAMILY_DEFAULT_FORM] > 0, fam_pred, np.inf)
    reg_family = regret(Tms[ntr:], FAMILY_DEFAULT_FORM[fam_pred.argmin(1)])
    report = {
        "train_loss_first": float(hist[0]), "train_loss_last": float(hist[-1]),
        "train_regret_mean": float(regret(Tms[:ntr], choose(pred_tr, Tms[:ntr])).mean()),
        "heldout": len(Fte),
        "selector_regret_mean": float(reg.mean()),
        "selector_regret_median": float(np.median(reg)),
        "selector_regret_p90": float(np.quantile(reg, 0.9)),
        "selector_top1": float((reg == 0).mean()),
        "fixed_form": FORM_NAMES[fixed],
        "fixed_regret_mean": float(reg_fixed.mean()),
        "variant_only_regret_mean": float(reg_family.mean()),
        "oracle_best_counts": np.bincount(np.argmin(np.where(Tms[ntr:] > 0, Tms[ntr:], np.inf), 1),
                                          minlength=_abi.NVARIANTS).tolist(),
        "selector_choice_counts": np.bincount(choice, minlength=_abi.NVARIANTS).tolist(),
    }
    return net, report


def main():
    p = argparse.ArgumentParser()
    p.add_argument("cmd", choices=["generate", "evaluate"])
    p.add_argument("--out", default="tests/golden/selector/selector_timings.npz")
    p.add_argument("--data", default="tests/golden/selector/selector_timings.npz")
    p.add_argument("--train", type=int, default=N_TRAIN)
    p.add_argument("--test", type=int, default=N_TEST)
    p.add_argument("--reps", type=int, default=5)
    p.add_argument("--epochs", type=int, default=3000)
    p.add_argument("--lr", type=float, default=3e-3)
    a = p.parse_args()
    _abi.check(_abi.gpu().pava_init(0))
    if a.cmd == "generate":
        t0 = time.time()
        d = build_dataset(a.train, a.test, a.reps)
        np.savez_compressed(a.out, **d)
        print(json.dumps({"written": a.out, "matrices": a.train + a.test,
                          "seconds": round(time.time() - t0, 1),
                          "nnz_total": int(d["nnz"].sum())}))
    else:
        d = dict(np.load(a.data))
        t0 = time.time()
        _, rep = train_selector(d, a.epochs, a.lr)
        rep["train_seconds"] = round(time.time() - t0, 2)
        print(json.dumps(rep))


if __name__ == "__main__":
    main()
