"""Resident models rebuilt from their exported fields (fastpls_b200_model_import):
predictions, scores and LDA labels of the rebuilt model equal the original's."""
import numpy as np
import pytest

from fastpls_b200 import api, workloads as W
from fastpls_b200._lib import FastplsError
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method", ["simpls", "opls"])
@pytest.mark.parametrize("scaling", ["centering", "autoscaling"])
def test_regression_round_trip(method, scaling):
    x, y = W.latent_regression(300, 120, 3, 4, 0.4, 81, dtype=np.float64)
    xt, yt = W.latent_regression(70, 120, 3, 4, 0.4, 82, dtype=np.float64)
    kw = {"north": 1} if method == "opls" else {}
    model = api.fit_resident(x, y, ncomp=6, method=method, scaling=scaling, **kw)
    fields = api.export_model(model, scores=False)
    copy = api.import_model(fields, scaling=scaling)
    pre = [1, 3, 6]
    assert np.array_equal(copy.predict_path(xt, pre), model.predict_path(xt, pre))
    assert np.array_equal(copy.project(xt, 6), model.project(xt, 6))
    assert np.array_equal(copy.response_sums(xt, yt, prefix=4), model.response_sums(xt, yt, prefix=4))
    for f in (0, 1, 3, 4, 5):
        assert np.array_equal(copy.export(f), model.export(f))
    ref = (O.simpls_fit(x, y, ncomp=6, scaling={"centering": 1, "autoscaling": 2}[scaling])
           if method == "simpls" else None)
    if ref is not None:
        assert O.rel_err(copy.predict_path(xt, [6])[0], O.simpls_predict(ref, xt, 6)) < 1e-10
    with pytest.raises(FastplsError):
        copy.export(6)          # needs the training predictors
    model.close()
    copy.close()


def test_classification_lda_round_trip():
    x, lab = W.latent_classification(400, 150, 4, 3, 0.5, 83, dtype=np.float64)
    xt, _ = W.latent_classification(120, 150, 4, 3, 0.5, 84, dtype=np.float64)
    model = api.fit_resident(x, labels=lab, classes=4, ncomp=5)
    fields = api.export_model(model)
    copy = api.import_model(fields, labels=lab)
    pre = [1, 2, 5]
    for lda in (False, True):
        assert np.array_equal(copy.classify_path(xt, pre, lda=lda, top=2),
                              model.classify_path(xt, pre, lda=lda, top=2))
        assert np.array_equal(copy.predict_path(xt, pre, lda=lda), model.predict_path(xt, pre, lda=lda))
    # without the training scores and labels the rebuilt model predicts but has no LDA
    bare = api.import_model(api.export_model(model, scores=False))
    assert np.array_equal(bare.classify_path(xt, pre), model.classify_path(xt, pre))
    with pytest.raises(FastplsError, match="LDA requires"):
        bare.classify_path(xt, pre, lda=True)
    for m in (model, copy, bare):
        m.close()


def test_fp32_round_trip_within_rounding():
    x, y = W.latent_regression(250, 90, 2, 4, 0.4, 85, dtype=np.float32)
    xt, _ = W.latent_regression(60, 90, 2, 4, 0.4, 86, dtype=np.float32)
    model = api.fit_resident(x, y, ncomp=4, precision=32)
    copy = api.import_model(api.export_model(model), precision=32)
    a = copy.predict_path(xt, [4]).astype(np.float64)
    b = model.predict_path(xt, [4]).astype(np.float64)
    assert O.rel_err(a, b) < 1e-5
    model.close()
    copy.close()


def test_import_rejects_unsupported_and_incomplete():
    x, y = W.latent_regression(120, 40, 2, 3, 0.4, 87, dtype=np.float64)
    model = api.fit_resident(x, y, ncomp=3)
    fields = api.export_model(model)
    with pytest.raises(ValueError):
        api.import_model(dict(fields, method="kernelpls"))
    bad = dict(fields, scale_x=np.zeros_like(fields["scale_x"]))
    with pytest.raises(FastplsError, match="invalid imported model fields"):
        api.import_model(bad)
    with pytest.raises(FastplsError, match="labels need the training scores"):
        api.import_model(dict(fields, scores=None, classification=True),
                         labels=np.ones(120, dtype=np.int32))
    model.close()
