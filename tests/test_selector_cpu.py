"""CPU side of the learned selector: the committed training set and the CPU restatement of
the network used as the oracle for the GPU kernels (no GPU needed)."""
import os

import numpy as np
import pytest

from oracle import selector_ref as R
from pava_b200 import _abi
from pava_b200 import selector as S

DATA = os.path.join(os.path.dirname(__file__), "golden", "selector", "selector_timings.npz")


def test_training_set_file():
    if not os.path.exists(DATA):
        pytest.fail("tests/golden/selector/selector_timings.npz is missing (python -m pava_b200.selector generate)")
    d = np.load(DATA)
    n = int(d["n_train"]) + int(d["n_test"])
    assert (int(d["n_train"]), int(d["n_test"])) == (2000, 200)
    assert d["features"].shape == (n, 12) and d["times_ms"].shape == (n, _abi.NVARIANTS)
    assert np.isfinite(d["features"]).all()
    sell = S.FORM_FAMILY == 6
    assert (d["times_ms"][:, ~sell] > 0).mean() > 0.99  # nearly every other form ran
    # SELL takes the stencils and banded matrices and refuses the heavy-tailed power laws
    took = (d["times_ms"][:, sell] > 0).all(1)
    assert took[d["family"] == 0].mean() > 0.9 and took[d["family"] == 2].mean() < 0.5
    assert np.all(np.bincount(d["family"], minlength=4) == n // 4)
    assert d["rows"].min() >= 1e4 - 1 and d["rows"].max() <= 1e7
    assert d["nnz"].min() >= 5e4 and d["nnz"].max() <= 1.1e8
    # matrix i's spec is a pure function of i
    for i in (0, 1, 2, 3, 1234):
        assert S.spec(i) == S.spec(i)
        assert S.spec(i)["family"] == d["family"][i]


def test_specs_cover_the_ranges():
    rows, fam = [], []
    for i in range(400):
        sp = S.spec(i)
        rows.append(sp["m"])
        fam.append(sp["family"])
    rows = np.array(rows)
    assert rows.min() >= 1e4 and rows.max() <= 1e7
    assert np.log10(rows).std() > 0.5
    assert np.all(np.bincount(fam) == 100)


def test_cpu_gradient_against_finite_differences():
    rng = np.random.default_rng(1)
    P = rng.normal(scale=0.3, size=R.NP)
    X = rng.normal(size=(50, 12))
    T = rng.normal(size=(50, R.OUT))
    mask = (rng.uniform(size=(50, R.OUT)) > 0.2).astype(float)
    loss, g = R.mlp_loss_grad(P, X, T, mask)
    for p in rng.choice(R.NP, 40, replace=False):
        h = 1e-6
        Pp, Pm = P.copy(), P.copy()
        Pp[p] += h
        Pm[p] -= h
        fd = (R.mlp_loss_grad(Pp, X, T, mask)[0] - R.mlp_loss_grad(Pm, X, T, mask)[0]) / (2 * h)
        assert abs(fd - g[p]) <= 1e-7 + 1e-5 * abs(g[p])


def test_regret_definition():
    t = np.array([[1.0, 2.0, 1.5, 4.0, 1.1, 3.0], [2.0, 1.0, -1.0, 1.0, 5.0, 2.0]])
    r = S.regret(t, np.array([4, 2]))
    assert np.isclose(r[0], 0.1) and np.isinf(r[1])   # a failed variant is never acceptable
    assert np.array_equal(S.regret(t, np.array([0, 1])), [0.0, 0.0])


def test_cpu_features_small():
    # 3 x 4: row 0 = cols {0, 1}, row 1 empty, row 2 = cols {1, 3, 20}
    rp = np.array([0, 2, 2, 5])
    ci = np.array([0, 1, 1, 3, 20])
    f = R.features(rp, ci, 40)
    assert np.isclose(f[0], np.log10(3)) and np.isclose(f[1], np.log10(5))
    assert np.isclose(f[5], 1 / 3)                     # one empty row
    assert np.isclose(f[7], 2 / 3)                     # two rows with 1..4 nonzeros
    assert np.isclose(f[10], (1 + 2) / 5)              # x lines: row 0 one, row 2 two
    assert np.isclose(f[9], 1.0)                       # all within 64 of the diagonal


def test_form_space_matches_the_library():
    """The 32 forms: pava_variant's formats and tile parameters, their kernel variant
    (pava_variant_family), and the names and families the selector reports use."""
    import ctypes
    from pava_b200 import _abi
    L = _abi.gpu()
    assert len(S.FORM_NAMES) == _abi.NVARIANTS == R.OUT == _abi.MLP_OUT
    seen = set()
    for v in range(_abi.NVARIANTS):
        f = ctypes.c_int()
        o = _abi.PavaOpts()
        assert L.pava_variant(v, ctypes.byref(f), ctypes.byref(o)) == 0
        assert L.pava_variant_family(v) == S.FORM_FAMILY[v]
        name = S.FORM_NAMES[v]
        idx = "auto" if o.index_mode == _abi.INDEX_AUTO else "i32"
        if f.value == _abi.FORMAT_CVR:
            assert name == f"cvr_s{o.steps}_{idx}"
        elif f.value == _abi.FORMAT_CSR5:
            w = "tiles_wave" if o.tiles_per_chunk == _abi.TILES_WAVE else "tiles_default"
            assert o.tiles_per_chunk in (0, _abi.TILES_WAVE)
            assert name == f"csr5_s{o.sigma}_{w}_{idx}"
        elif f.value == _abi.FORMAT_SELL:
            assert name == f"sell_{idx}"
        else:
            assert f.value == _abi.FORMAT_CSR
            groups = o.rows_per_tile // (32 // o.lanes_per_row)
            assert name == f"csr_l{o.lanes_per_row}_g{groups}"
        key = (f.value, o.steps, o.sigma, o.tiles_per_chunk, o.index_mode, o.lanes_per_row,
               o.rows_per_tile)
        assert key not in seen
        seen.add(key)
    assert L.pava_variant(_abi.NVARIANTS, None, None) == _abi.E_INVALID_ARG
    assert L.pava_variant_family(-1) == -1
    for fam, v in enumerate(S.FAMILY_DEFAULT_FORM):
        assert S.FORM_FAMILY[v] == fam
