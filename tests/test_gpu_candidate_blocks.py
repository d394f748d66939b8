"""Candidate blocks of SIMPLS directions on the device vs the FP64 oracle.

Classification fits with n p q >= 5e8, q <= 2048 and at least 4 components take
min(64, components, p, q) directions from one decomposition of the
cross-product (src/cuda_resident_simpls.cuh:144-190): the single fit, each
CV fold fit, and the inner SIMPLS of OPLS and kernel PLS
(src/cuda_resident_special.cuh:315, :492)."""
import numpy as np
import pytest

from fastpls_b200 import api, workloads as W
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu

Q = 50


def _data(n, p, seed):
    return W.latent_classification(n, p, Q, 50, 0.5, seed, dtype=np.float64)


@pytest.mark.parametrize("precision", [64, 32])
def test_simpls_block_fit(precision):
    n, p, a = 4000, 2500, 8
    x, lab = _data(n, p, 61)
    xt, _ = _data(300, p, 62)
    assert O.simpls_block_size(n, p, Q, a, True) == a
    if precision == 32:
        x = x.astype(np.float32).astype(np.float64)
        xt = xt.astype(np.float32).astype(np.float64)
    model = api.fit_resident(x, labels=lab, classes=Q, ncomp=a, precision=precision)
    ref = O.simpls_fit(x, labels=lab, classes=Q, ncomp=a, scaling=1)
    pre = [1, 3, 4, 8]
    pred = model.predict_path(xt, pre).astype(np.float64)
    tol = 1e-9 if precision == 64 else 2e-5
    for j, k in enumerate(pre):
        assert O.rel_err(pred[j], O.simpls_predict(ref, xt, k)) < tol
    if precision == 64:
        got = model.classify_path(xt, pre, top=1)
        for j, k in enumerate(pre):
            assert np.array_equal(got[j][:, 0], O.row_argmax(O.simpls_predict(ref, xt, k)))
        R = model.export(0)
        assert O.rel_err(O.align_signs(R, ref["R"]), ref["R"]) < 1e-9
    model.close()


def test_cv_classification_block_folds():
    n, p = 5000, 3000
    x, lab = _data(n, p, 63)
    folds = W.uneven_folds(n, 5, 63)
    pre = [1, 4, 6]
    for f in range(1, 6):
        assert O.simpls_block_size(int((folds != f).sum()), p, Q, 6, True) == 6
    got = api.cv_classification(x, lab, Q, folds, pre, store_predictions=True)
    ref = O.cv_classification(x, lab, Q, folds, pre, store_predictions=True)
    assert np.array_equal(got["predictions"], ref["predictions"])
    assert np.allclose(got["metrics"], ref["metrics"])


def test_opls_classification_block():
    n, p, a = 4000, 2500, 6
    x, lab = _data(n, p, 64)
    xt, _ = _data(200, p, 65)
    model = api.fit_resident(x, labels=lab, classes=Q, ncomp=a, method="opls", north=1)
    ref = O.opls_fit(x, labels=lab, classes=Q, ncomp=a, north=1)
    pred = model.predict_path(xt, [2, 6])
    for j, k in enumerate([2, 6]):
        assert O.rel_err(pred[j], O.opls_predict(ref, xt, k)) < 1e-9
    model.close()


def test_kernelpls_classification_block():
    n, p, a = 3200, 120, 6
    x, lab = _data(n, p, 66)
    xt, _ = _data(150, p, 67)
    assert O.simpls_block_size(n, n, Q, a, True) == a
    model = api.fit_resident(x, labels=lab, classes=Q, ncomp=a, method="kernelpls",
                             kernel="rbf", gamma=1e-4)
    ref = O.kernelpls_fit(x, labels=lab, classes=Q, ncomp=a, kind=2, gamma=1e-4)
    pred = model.predict_path(xt, [3, 6])
    for j, k in enumerate([3, 6]):
        assert O.rel_err(pred[j], O.kernelpls_predict(ref, xt, k)) < 1e-9
    model.close()


def test_massive_fp32_regression_cross_covariance():
    """FP32 regression whose p x q cross-covariance exceeds 512 MiB (4.2e6 x
    33 x 4 bytes = 554 MB): the regime where the reference switches to its
    implicit cross-covariance route and to blocks of min(8, a, p, q)
    candidates (src/cuda_resident_simpls.cuh:125-127, :133-153). The device
    keeps S explicit (1.1 GB in FP64) and takes the same candidate blocks;
    coefficients and predictions match the FP64 oracle run with that block
    rule on the same FP32-rounded values."""
    n, p, q, a = 40, 4_200_000, 33, 10
    assert p * q * 4 > 512 * 1024 * 1024
    x, y = W.latent_regression(n, p, q, 6, 0.5, 71, dtype=np.float32)
    block = O.simpls_block_size(n, p, q, a, False, fp32=True)
    assert block == 8
    model = api.fit_resident(x, y, ncomp=a, precision=32)
    R = model.export(0).astype(np.float64)
    Qm = model.export(1).astype(np.float64)
    pre = [1, 8, 10]
    pred = model.predict_path(x[:20], pre).astype(np.float64)
    model.close()
    x64 = x.astype(np.float64)
    del x
    ref = O.simpls_fit(x64, y.astype(np.float64), ncomp=a, scaling=1, block=block)
    for k in pre:
        assert O.rel_err(R[:, :k] @ Qm[:, :k].T, ref["R"][:, :k] @ ref["Q"][:, :k].T) < 1e-7, k
    for j, k in enumerate(pre):
        assert O.rel_err(pred[j], O.simpls_predict(ref, x64[:20], k)) < 1e-7, k


def test_block_wider_than_the_rank_completes():
    """A classification block of q classes is one wider than the rank q - 1
    of the centred label cross-product: the last candidate of the block has a
    numerically zero eigenvalue. The fit completes (as the reference's does,
    with whatever unit direction its sketch gives there), and every prefix
    within the rank matches the oracle."""
    n, p, q, a = 4000, 25000, 6, 8
    x, lab = W.latent_classification(n, p, q, 5, 0.5, 73, dtype=np.float64)
    present = np.unique(lab)
    assert present.size == q
    assert O.simpls_block_size(n, p, q, a, True) == q
    model = api.fit_resident(x, labels=lab, classes=q, ncomp=a, precision=64)
    assert model.controls()["block"] == q
    xt, _ = W.latent_classification(300, p, q, 5, 0.5, 74, dtype=np.float64)
    pre = [1, 3, q - 1]
    pred = model.predict_path(xt, pre).astype(np.float64)
    ref = O.simpls_fit(x, labels=lab, classes=q, ncomp=a, scaling=1)
    for j, k in enumerate(pre):
        assert O.rel_err(pred[j], O.simpls_predict(ref, xt, k)) < 1e-8, k
    assert np.all(np.isfinite(model.export(0)))
    model.close()
