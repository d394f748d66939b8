"""OPLS and nonlinear kernel PLS through the C ABI vs the FP64 oracle.

The reference pins CUDA vs CPU predictions for these at 1e-10 relative in
FP64 (tests/testthat/test-cuda-resident-public.R:125-168)."""
import numpy as np
import pytest

from fastpls_b200 import api, workloads as W
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("north", [0, 1, 2])
@pytest.mark.parametrize("scaling", [1, 2])
def test_opls_predictions(north, scaling):
    x, y = W.latent_regression(160, 90, 3, 4, 0.5, 51, dtype=np.float64)
    xt, _ = W.latent_regression(40, 90, 3, 4, 0.5, 52, dtype=np.float64)
    model = api.fit_resident(x, y, ncomp=4, scaling=scaling, method="opls", north=north)
    ref = O.opls_fit(x, y, ncomp=4, scaling=scaling, north=north)
    pred = model.predict_path(xt, [1, 2, 4])
    for j, k in enumerate([1, 2, 4]):
        assert O.rel_err(pred[j], O.opls_predict(ref, xt, k)) < 1e-10
    R = model.export(0)
    assert O.rel_err(O.align_signs(R, ref["R_eff"]), ref["R_eff"]) < 1e-9
    model.close()


@pytest.mark.parametrize("kernel,gamma,degree", [("rbf", 0.015, 3), ("poly", 0.01, 2)])
def test_kernelpls_predictions(kernel, gamma, degree):
    x, y = W.latent_regression(150, 70, 2, 4, 0.5, 53, dtype=np.float64)
    xt, _ = W.latent_regression(37, 70, 2, 4, 0.5, 54, dtype=np.float64)
    model = api.fit_resident(x, y, ncomp=5, method="kernelpls", kernel=kernel,
                             gamma=gamma, degree=degree, coef0=1.0)
    kind = {"rbf": 2, "poly": 3}[kernel]
    ref = O.kernelpls_fit(x, y, ncomp=5, kind=kind, gamma=gamma, degree=degree, coef0=1.0)
    pred = model.predict_path(xt, [2, 5])
    for j, k in enumerate([2, 5]):
        assert O.rel_err(pred[j], O.kernelpls_predict(ref, xt, k)) < 1e-10
    assert model.export(0).shape == (150, 5)      # feature_p = n
    assert model.export(3).shape == (70,)         # input centring stays p-long
    model.close()


def test_opls_classification_lda_runs():
    x, lab = W.latent_classification(200, 60, 3, 3, 0.5, 55, dtype=np.float64)
    model = api.fit_resident(x, labels=lab, classes=3, ncomp=3, method="opls", north=1)
    got = model.classify_path(x, [1, 3], lda=True)
    assert got.shape == (2, 200, 1) and got.min() >= 1 and got.max() <= 3
    assert (got[1][:, 0] == lab).mean() > 0.8
    model.close()
