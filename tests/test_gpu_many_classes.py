"""Classification with many classes (65-112, beyond one warp's Jacobi and a
64-bit class mask): SIMPLS with LDA, PLS-SVD and CV against the oracle."""
import numpy as np
import pytest

from fastpls_b200 import api, workloads as W
from fastpls_b200._lib import FastplsError
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu

CLASSES = 100


def _data(n, p, seed):
    x, lab = W.latent_classification(n, p, CLASSES, 60, 0.5, seed, dtype=np.float64)
    assert np.bincount(lab, minlength=CLASSES + 1)[1:].min() > 0
    return x, lab


def test_simpls_many_classes_lda():
    x, lab = _data(4000, 150, 111)
    xt, _ = _data(4000, 150, 112)
    xt = xt[:300]
    model = api.fit_resident(x, labels=lab, classes=CLASSES, ncomp=6)
    ref = O.simpls_fit(x, labels=lab, classes=CLASSES, ncomp=6)
    pre = [1, 3, 6]
    pred = model.predict_path(xt, pre)
    for j, k in enumerate(pre):
        assert O.rel_err(pred[j], O.simpls_predict(ref, xt, k)) < 1e-9
    got = model.classify_path(xt, pre, lda=True)
    lda = O.lda_train(ref["T"], lab, CLASSES, pre)
    tt = O.simpls_project(ref, xt, 6)
    for j in range(len(pre)):
        assert np.array_equal(got[j][:, 0], O.row_argmax(O.lda_discriminants(lda[j], tt)))
    model.close()


def test_plssvd_many_classes():
    x, lab = _data(4000, 150, 113)
    model = api.fit_resident(x, labels=lab, classes=CLASSES, ncomp=5, method="plssvd")
    ref = O.plssvd_fit(x, labels=lab, classes=CLASSES, prefixes=[1, 3, 5])
    pred = model.predict_path(x[:200], [1, 3, 5])
    for j in range(3):
        assert O.rel_err(pred[j], O.plssvd_predict(ref, x[:200], j)) < 1e-9
    model.close()


def test_response_limit():
    x = np.random.default_rng(1).standard_normal((200, 20))
    lab = (np.arange(200) % 113 + 1).astype(np.int32)
    with pytest.raises(FastplsError, match="1..112"):
        api.fit_resident(x, labels=lab, classes=113, ncomp=2)
