"""Host side of the SELL form (no GPU): the stored-element count of its slices and the padding
rule pava_create applies (matrices.sell_padded_elements / sell_accepts), on hand-counted
matrices, and the form's place in the library's form space."""
import numpy as np

from pava_b200 import _abi
from pava_b200 import matrices as M
from pava_b200 import selector as S


def _lens(lens, n=1000):
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.arange(L) for L in lens]).astype(np.int32) if rp[-1] else \
        np.zeros(0, np.int32)
    return M.from_arrays(len(lens), n, rp, ci, np.ones(int(rp[-1])))


def test_padded_elements_hand_counted():
    # one slice: the longest row (5) rounds up to 8, 32 lanes x 8
    assert M.sell_padded_elements(_lens([5] + [1] * 31)) == 256
    # rows of exactly 4: one block per slice, no padding inside it
    assert M.sell_padded_elements(_lens([4] * 64)) == 2 * 128
    # 33 rows: the second slice holds one row and 31 absent ones, padded all the same
    assert M.sell_padded_elements(_lens([6] * 33)) == 2 * 256
    # empty slices store nothing
    assert M.sell_padded_elements(_lens([0] * 32 + [3] * 32)) == 128
    assert M.sell_padded_elements(_lens([0] * 10)) == 0


def test_accepts_rule():
    # stored <= 2 nnz + 128 per slice
    assert M.sell_accepts(_lens([4] + [1] * 31))        # 128 <= 2 * 35 + 128
    assert not M.sell_accepts(_lens([5] + [1] * 31))    # 256 > 2 * 36 + 128
    assert M.sell_accepts(_lens([27] * 64))             # 28 / 27 padding
    assert M.sell_accepts(_lens([0] * 100))             # nothing stored
    # the benchmark matrices: the stencil and the band are taken, the power law refused
    assert M.sell_accepts(M.stencil27(20))
    assert M.sell_accepts(M.banded(10_000, 64, 24))
    assert not M.sell_accepts(M.powerlaw(50_000, seed=1))


def test_padding_ratio_of_the_stencil_and_laplacian():
    A = M.stencil27(40)
    assert 1.0 < M.sell_padded_elements(A) / A.nnz < 1.1   # 27 -> 28, shorter boundary rows
    L = M.laplace2d(64)
    assert 1.5 < M.sell_padded_elements(L) / L.nnz < 1.7   # 5 -> 8


def test_sell_in_the_form_space():
    assert _abi.FORMAT_SELL == 4
    sell = [v for v in range(_abi.NVARIANTS) if S.FORM_FAMILY[v] == 6]
    assert [S.FORM_NAMES[v] for v in sell] == ["sell_i32", "sell_auto"]
    assert S.FAMILY_NAMES[6] == "sell" and S.FORM_FAMILY[S.FAMILY_DEFAULT_FORM[6]] == 6


def test_choose_skips_forms_that_refuse():
    """The selection rule: the smallest prediction among the forms that took the matrix."""
    pred = np.array([[0.1, 0.5, 0.2], [0.3, 0.2, 0.9]])
    times = np.array([[-1.0, 2.0, 3.0], [1.0, 2.0, 3.0]])   # form 0 refused matrix 0
    assert S.choose(pred, times).tolist() == [2, 1]
