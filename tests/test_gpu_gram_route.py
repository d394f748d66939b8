"""The cached predictor cross-product route of classification SIMPLS
(src/cuda_resident_simpls.cuh:135, src/cuda_resident_component.cuh:131-167):
with labels, at least 8 components and n >= 8 p the loadings come from the
p x p Gram of the standardised predictors. The model must equal the FP64
oracle (the same mathematics as the per-pass route), and the controls must
report the route."""
import numpy as np
import pytest

from fastpls_b200 import api, workloads as W
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,scaling", [(64, 1), (64, 2), (32, 1), (64, 3)])
def test_gram_route_fit_matches_oracle(precision, scaling):
    n, p, classes, a = 3000, 300, 4, 10
    x, lab = W.latent_classification(n, p, classes, 5, 0.5, 81, dtype=np.float64)
    xt, _ = W.latent_classification(200, p, classes, 5, 0.5, 82, dtype=np.float64)
    if precision == 32:
        x = x.astype(np.float32).astype(np.float64)
        xt = xt.astype(np.float32).astype(np.float64)
    model = api.fit_resident(x, labels=lab, classes=classes, ncomp=a, precision=precision,
                             scaling=scaling)
    ctl = model.controls()
    assert ctl["predictor_crossprod_cache"] == 1 and ctl["block"] == 1, ctl
    ref = O.simpls_fit(x, labels=lab, classes=classes, ncomp=a, scaling=scaling)
    R = model.export(0)
    T = model.export(2)
    tol = 1e-9 if precision == 64 else 1e-6
    assert O.rel_err(O.align_signs(R, ref["R"]), ref["R"]) < tol
    assert O.rel_err(O.align_signs(T, ref["T"]), ref["T"]) < tol
    pre = [1, 4, 10]
    pred = model.predict_path(xt, pre).astype(np.float64)
    for j, k in enumerate(pre):
        assert O.rel_err(pred[j], O.simpls_predict(ref, xt, k)) < tol
    if precision == 64:
        got = model.classify_path(xt, pre, lda=True)
        lda = O.lda_train(ref["T"], lab, classes, pre)
        tt = O.simpls_project(ref, xt, a)
        for j, k in enumerate(pre):
            want = O.row_argmax(O.lda_discriminants(lda[j], tt[:, :k]))
            assert np.array_equal(got[j][:, 0], want), k
    model.close()


def test_gram_route_not_taken_for_regression_or_wide_data():
    x, y = W.latent_regression(3000, 300, 3, 5, 0.5, 83, dtype=np.float64)
    m = api.fit_resident(x, y, ncomp=10, precision=64)
    assert m.controls()["predictor_crossprod_cache"] == 0
    m.close()
    x, lab = W.latent_classification(1000, 300, 3, 5, 0.5, 84, dtype=np.float64)
    m = api.fit_resident(x, labels=lab, classes=3, ncomp=10, precision=64)
    assert m.controls()["predictor_crossprod_cache"] == 0   # n < 8 p
    m.close()


def test_gram_route_classification_cv_matches_oracle():
    n, p, classes = 2400, 250, 3
    x, lab = W.latent_classification(n, p, classes, 5, 0.5, 85, dtype=np.float64)
    folds = W.uneven_folds(n, 4, 85)
    pre = [1, 5, 9]
    got = api.cv_classification(x, lab, classes, folds, pre, precision=64)
    want = O.cv_classification(x, lab, classes, folds, pre)
    assert np.array_equal(got["metrics"], want["metrics"]), (got["metrics"], want["metrics"])
