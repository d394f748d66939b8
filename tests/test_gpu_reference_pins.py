"""Pins the reference's own R tests hold for the CUDA path, restated on the C ABI:
tests/testthat/test-cuda-resident-public.R:73-104 (the classification path
equals independent per-prefix prediction exactly), test-cuda-simpls-compact-
prediction.R:1-38 (compaction keeps R, Q and predictions bitwise),
test-core-dense-regression.R:1-33 (fit-time predictions equal predict() on the
training rows to 1e-10) and test-core-cv-parity.R:1-120 (FP32 vs FP64 CV
within 1e-4, identical class predictions)."""
import numpy as np
import pytest

from fastpls_b200 import api, workloads as W
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method", ["simpls", "plssvd"])
@pytest.mark.parametrize("lda", [False, True])
def test_classification_path_equals_per_prefix(method, lda):
    x, lab = W.latent_classification(300, 80, 5, 4, 0.5, 101, dtype=np.float64)
    xt, _ = W.latent_classification(90, 80, 5, 4, 0.5, 102, dtype=np.float64)
    model = api.fit_resident(x, labels=lab, classes=5, ncomp=4, method=method)
    pre = [1, 2, 3, 4]
    path, resp = model.classify_path(xt, pre, lda=lda, top=3, responses=True)
    for j, k in enumerate(pre):
        one, one_resp = model.classify_path(xt, [k], lda=lda, top=3, responses=True)
        assert np.array_equal(path[j], one[0])
        assert np.array_equal(resp[j], one_resp[0])
    model.close()


@pytest.mark.parametrize("precision", [64, 32])
def test_compaction_keeps_model_and_predictions(precision):
    x, lab = W.latent_classification(280, 90, 3, 3, 0.5, 103, dtype=np.float64)
    xt, _ = W.latent_classification(60, 90, 3, 3, 0.5, 104, dtype=np.float64)
    model = api.fit_resident(x, labels=lab, classes=3, ncomp=3, precision=precision)
    before = (model.export(0), model.export(1), model.predict_path(xt, [1, 3]),
              model.classify_path(xt, [1, 3], lda=True))
    model.compact(prepare_lda=True)
    after = (model.export(0), model.export(1), model.predict_path(xt, [1, 3]),
             model.classify_path(xt, [1, 3], lda=True))
    for b, a in zip(before, after):
        assert np.array_equal(b, a)
    model.close()


def test_fit_time_predictions_equal_predict():
    x, y = W.latent_regression(200, 60, 2, 3, 0.3, 105, dtype=np.float64)
    model = api.fit_resident(x, y, ncomp=4)
    T, Q, ym = model.export(2), model.export(1), model.export(5)
    fitted = ym + T @ Q.T
    assert O.rel_err(model.predict_path(x, [4])[0], fitted) < 1e-10
    model.close()


def test_cv_fp32_vs_fp64():
    x, y = W.latent_regression(240, 100, 2, 4, 0.4, 106, dtype=np.float64)
    folds = W.uneven_folds(240, 6, 106)
    pre = [1, 2, 4, 6]
    a = api.cv_regression(x, y, folds, pre, precision=64)
    b = api.cv_regression(x.astype(np.float32), y.astype(np.float32), folds, pre, precision=32)
    assert np.allclose(a["q2"], b["q2"], rtol=1e-4, atol=1e-6)
    xc, lab = W.latent_classification(240, 100, 3, 4, 0.5, 107, dtype=np.float64)
    c = api.cv_classification(xc, lab, 3, folds, pre, precision=64, store_predictions=True)
    d = api.cv_classification(xc.astype(np.float32), lab, 3, folds, pre, precision=32,
                              store_predictions=True)
    assert np.array_equal(c["predictions"], d["predictions"])
    assert np.allclose(c["metrics"], d["metrics"])


def test_label_crossprod_known_answer_on_device():
    # core/tests/test_core_classification.cpp:13-44 through a PLS-SVD fit: the
    # autoscaled label cross-product is a = 0.7745967 times [-1, 1] in every
    # row, so the weight is (1, 1, 1) / sqrt(3) up to sign
    x = np.array([[1 + r + 10 * c for c in range(3)] for r in range(4)], dtype=np.float64)
    lab = np.array([1, 2, 1, 2], dtype=np.int32)
    model = api.fit_resident(x, labels=lab, classes=2, ncomp=1, method="plssvd",
                             scaling="autoscaling")
    assert np.allclose(model.export(3), [2.5, 12.5, 22.5], atol=1e-12)
    assert np.allclose(model.export(4), 1.2909944, atol=1e-6)
    assert np.allclose(model.export(5), [0.5, 0.5], atol=1e-12)
    R = model.export(0)[:, 0]
    assert np.allclose(np.abs(R), 1 / np.sqrt(3), atol=1e-12)
    assert np.all(np.sign(R) == np.sign(R[0]))
    model.close()
