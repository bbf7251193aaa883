"""Kernel-matrix blocks (svmb_rows_kernel_block) in the three arithmetic forms
against a float64 numpy restatement of the reference's kernels
(reference libsvm/svm.cpp:235-254, dot products :305-325).

Tolerances, per output, with S = sum_k |a_k b_k| and u = 2^-24:
  exact   |dK| <= 1e-12 (1 + |K|)              float64 accumulation
  fp32    |d dot| <= d u S                     sequential float32 accumulation
  bf16x3  |d dot| <= (2^-14 + 2 d u) S         bf16 split products (~2^-16 each), float32 accumulation
  fp16x3  |d dot| <= (2^-19 + 2 d u) M         scaled fp16 split (~2^-22 of the row maxima), M = d max|a| max|b|
  tf32    |d dot| <= (2^-10 + 2 d u) S         inputs rounded to tf32 (2^-11 each), float32 accumulation
RBF values are held to |dK| <= K * gamma * 2 * (dot bound + norm bound)."""
import numpy as np
import pytest

from svmb200 import datagen
from svmb200.lib import FORM_BF16X3, FORM_EXACT, FORM_FP16X3, FORM_FP32, FORM_TF32, ResidentRows, make_params

pytestmark = pytest.mark.gpu


def _dense_rows(n, d, seed, zero_frac=0.0):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, d)).astype(np.float32)
    if zero_frac:
        X[rng.random((n, d)) < zero_frac] = 0.0
    y = np.where(rng.random(n) < 0.5, 1.0, -1.0)
    return datagen.from_dense(X, y), X.astype(np.float64)


def _blocks(n, ma, nb, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(0, n, ma).astype(np.int32), rng.integers(0, n, nb).astype(np.int32)


@pytest.mark.parametrize("n,d,ma,nb", [(300, 100, 200, 150), (1000, 784, 300, 260), (64, 8, 1, 1)])
def test_linear_block_forms(engine, n, d, ma, nb):
    p, X = _dense_rows(n, d, seed=n + d)
    rows = ResidentRows(engine, p)
    assert rows.dense
    ia, ib = _blocks(n, ma, nb, seed=d)
    A, B = X[ia], X[ib]
    want = A @ B.T
    S = np.abs(A) @ np.abs(B).T
    u = 2.0 ** -24
    forms = (FORM_EXACT, FORM_FP32, FORM_BF16X3, FORM_FP16X3, FORM_TF32)
    got = {f: rows.kernel_block(ia, ib, make_params(kernel_type=0, form=f)) for f in forms}
    rel = {f: float((np.abs(got[f] - want) / S).max()) for f in got}
    M = d * np.abs(A).max(1)[:, None] * np.abs(B).max(1)[None, :]
    assert np.all(np.abs(got[FORM_FP16X3] - want) <= (2.0 ** -19 + 2 * d * u) * M + 1e-30), rel
    assert np.all(np.abs(got[FORM_EXACT] - want) <= 1e-12 * (1 + np.abs(want))), rel
    assert np.all(np.abs(got[FORM_FP32] - want) <= d * u * S + 1e-30), rel
    assert np.all(np.abs(got[FORM_BF16X3] - want) <= (2.0 ** -14 + 2 * d * u) * S + 1e-30), rel
    assert np.all(np.abs(got[FORM_TF32] - want) <= (2.0 ** -10 + 2 * d * u) * S + 1e-30), rel
    # the split form is far more accurate than a single bf16 product (2^-8)
    assert rel[FORM_BF16X3] < 2.0 ** -12, rel
    # and a single tf32 product is less accurate than either split form
    assert rel[FORM_TF32] > rel[FORM_BF16X3], rel


def test_rbf_block_tensor_form(engine):
    n, d, gamma = 2000, 784, 1.0 / 784
    tr, _ = datagen.dense_pixels(n=n, n_test=0, d=d)
    X = tr.to_dense().astype(np.float64)
    rows = ResidentRows(engine, tr, layout=1)
    ia, ib = _blocks(n, 257, 513, seed=5)
    A, B = X[ia], X[ib]
    sq = (X * X).sum(1)
    dot = A @ B.T
    want = np.exp(-gamma * (sq[ia][:, None] + sq[ib][None, :] - 2 * dot))
    S = np.abs(A) @ np.abs(B).T
    got = rows.kernel_block(ia, ib, make_params(kernel_type=2, gamma=gamma, form=FORM_BF16X3))
    u = 2.0 ** -24
    bound = want * gamma * 2 * ((2.0 ** -14 + 2 * d * u) * S + 1e-12 * (sq[ia][:, None] + sq[ib][None, :])) + 1e-12
    assert np.all(np.abs(got - want) <= bound)
    got16 = rows.kernel_block(ia, ib, make_params(kernel_type=2, gamma=gamma, form=FORM_FP16X3))
    M = d * np.abs(A).max(1)[:, None] * np.abs(B).max(1)[None, :]
    bound16 = want * gamma * 2 * ((2.0 ** -19 + 2 * d * u) * M + 1e-12 * (sq[ia][:, None] + sq[ib][None, :])) + 1e-12
    assert np.all(np.abs(got16 - want) <= bound16)
    # the scaled fp16 split is the more accurate one
    assert np.abs(got16 - want).max() < np.abs(got - want).max()
    ex = rows.kernel_block(ia, ib, make_params(kernel_type=2, gamma=gamma, form=FORM_EXACT))
    assert np.all(np.abs(ex - want) <= 1e-12)


def test_tensor_form_on_csr_rows(engine):
    """CSR-resident rows are scattered into the dense split copy."""
    p, _ = datagen.sparse_text(n=300, n_test=0, d=5000)
    rows = ResidentRows(engine, p)
    assert not rows.dense
    X = p.to_dense().astype(np.float64)
    ia, ib = _blocks(p.n, 130, 70, seed=9)
    want = X[ia] @ X[ib].T
    S = np.abs(X[ia]) @ np.abs(X[ib]).T
    got = rows.kernel_block(ia, ib, make_params(kernel_type=0, form=FORM_BF16X3))
    assert np.all(np.abs(got - want) <= (2.0 ** -14 + 2 * 5000 * 2.0 ** -24) * S + 1e-30)
    got16 = rows.kernel_block(ia, ib, make_params(kernel_type=0, form=FORM_FP16X3))
    M = 5000 * np.abs(X[ia]).max(1)[:, None] * np.abs(X[ib]).max(1)[None, :]
    assert np.all(np.abs(got16 - want) <= (2.0 ** -19 + 2 * 5000 * 2.0 ** -24) * M + 1e-30)
    got32 = rows.kernel_block(ia, ib, make_params(kernel_type=0, form=FORM_TF32))
    assert np.all(np.abs(got32 - want) <= (2.0 ** -10 + 2 * 5000 * 2.0 ** -24) * S + 1e-30)
    ex = rows.kernel_block(ia, ib, make_params(kernel_type=0, form=FORM_EXACT))
    assert np.all(np.abs(ex - want) <= 1e-12 * (1 + np.abs(want)))


@pytest.mark.parametrize("form", [FORM_FP16X3, FORM_BF16X3, FORM_TF32])
def test_many_tiles_per_cta_one_chunk(engine, form):
    """d <= 64: one 64-feature chunk per 128 x 64 tile, so the persistent
    CTAs walk ~15 tiles each and the tile ring of column data wraps twice;
    ragged block edges.  Same bounds as the linear-block test."""
    n, d = 6000, 40
    p, X = _dense_rows(n, d, seed=11)
    rows = ResidentRows(engine, p)
    ia, ib = _blocks(n, 3001, 6003, seed=12)
    A, B = X[ia], X[ib]
    want = A @ B.T
    S = np.abs(A) @ np.abs(B).T
    u = 2.0 ** -24
    got = rows.kernel_block(ia, ib, make_params(kernel_type=0, form=form))
    if form == FORM_FP16X3:
        M = d * np.abs(A).max(1)[:, None] * np.abs(B).max(1)[None, :]
        bound = (2.0 ** -19 + 2 * d * u) * M
    elif form == FORM_BF16X3:
        bound = (2.0 ** -14 + 2 * d * u) * S
    else:
        bound = (2.0 ** -10 + 2 * d * u) * S
    assert np.all(np.abs(got - want) <= bound + 1e-30)
