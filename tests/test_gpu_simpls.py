"""SIMPLS / PLS-SVD single fits through the C ABI vs the FP64 oracle."""
import numpy as np
import pytest

from fastpls_b200 import api, workloads as W
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-9   # FP64 arithmetic on the device vs the FP64 oracle
TOL_B = 1e-8   # coefficient matrices (products of sign-aligned factors)


def _fit_case(precision, scaling, ncomp=10, n=500, p=2000, m=3):
    dt = np.float64 if precision == 64 else np.float32
    x, y = W.latent_regression(n, p, m, 5, 0.5, 1, dtype=dt)
    xt, _ = W.latent_regression(120, p, m, 5, 0.5, 11, dtype=dt)
    model = api.fit_resident(x, y, ncomp=ncomp, scaling=scaling,
                             precision=precision)
    ref = O.simpls_fit(x.astype(np.float64), y.astype(np.float64),
                       ncomp=ncomp, scaling=scaling)
    return x, y, xt, model, ref


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("scaling", [1, 2, 3])
def test_simpls_plain_config(precision, scaling):
    """500 x 2000, m = 3, ncomp = 10 (plain SIMPLS configuration)."""
    x, y, xt, model, ref = _fit_case(precision, scaling)
    R = model.export(0).astype(np.float64)
    Q = model.export(1).astype(np.float64)
    T = model.export(2).astype(np.float64)
    tol = TOL64 if precision == 64 else 2e-6  # FP32 outputs are rounded
    assert O.rel_err(O.align_signs(R, ref["R"]), ref["R"]) < tol
    assert O.rel_err(O.align_signs(T, ref["T"]), ref["T"]) < tol
    B, Bref = R @ Q.T, ref["R"] @ ref["Q"].T
    assert O.rel_err(B, Bref) < (TOL_B if precision == 64 else 2e-6)
    assert np.allclose(model.export(3), ref["centre"], rtol=1e-6, atol=1e-6)
    assert np.allclose(model.export(5), ref["ymean"], rtol=1e-6, atol=1e-6)
    pre = list(range(1, 11))
    pred = model.predict_path(xt, pre).astype(np.float64)
    for j, a in enumerate(pre):
        want = O.simpls_predict(ref, xt.astype(np.float64), a)
        assert O.rel_err(pred[j], want) < (TOL_B if precision == 64 else 2e-6)
    sc = model.project(xt, 4).astype(np.float64)
    want = O.simpls_project(ref, xt.astype(np.float64), 4)
    assert O.rel_err(O.align_signs(sc, want), want) < (TOL64 if precision == 64 else 2e-6)
    model.close()


def test_simpls_classification_lda():
    x, lab = W.latent_classification(400, 300, 4, 3, 0.5, 5, dtype=np.float64)
    xt, labt = W.latent_classification(150, 300, 4, 3, 0.5, 6, dtype=np.float64)
    model = api.fit_resident(x, labels=lab, classes=4, ncomp=6, precision=64)
    ref = O.simpls_fit(x, labels=lab, classes=4, ncomp=6, scaling=1)
    pre = [1, 2, 4, 6]
    got = model.classify_path(xt, pre, lda=False, top=1)
    got_lda = model.classify_path(xt, pre, lda=True, top=1)
    ttest = O.simpls_project(ref, xt, 6)
    ldas = O.lda_train(ref["T"], lab, 4, pre)
    for j, a in enumerate(pre):
        yh = O.simpls_predict(ref, xt, a)
        assert np.array_equal(got[j][:, 0], O.row_argmax(yh))
        d = O.lda_discriminants(ldas[j], ttest)
        assert np.array_equal(got_lda[j][:, 0], O.row_argmax(d))
    disc = model.predict_path(xt, pre, lda=True)
    for j in range(len(pre)):
        d = O.lda_discriminants(ldas[j], ttest)
        assert O.rel_err(disc[j], d) < 1e-9
    model.close()


@pytest.mark.parametrize("classify", [False, True])
def test_plssvd(classify):
    if classify:
        x, lab = W.latent_classification(300, 250, 5, 4, 0.3, 7, dtype=np.float64)
        model = api.fit_resident(x, labels=lab, classes=5, ncomp=4, method="plssvd")
        ref = O.plssvd_fit(x, labels=lab, classes=5, prefixes=[1, 2, 3, 4])
    else:
        x, y = W.latent_regression(300, 250, 6, 4, 0.3, 8, dtype=np.float64)
        model = api.fit_resident(x, y, ncomp=4, method="plssvd")
        ref = O.plssvd_fit(x, y, prefixes=[1, 2, 3, 4])
    R = model.export(0)
    assert O.rel_err(O.align_signs(R, ref["R"]), ref["R"]) < 1e-9
    pred = model.predict_path(x, [1, 2, 3, 4])
    for j in range(4):
        assert O.rel_err(pred[j], O.plssvd_predict(ref, x, j)) < 1e-9
    model.close()


@pytest.mark.parametrize("m,k,n", [(256, 300, 190), (130, 78, 211), (384, 64, 128),
                                   (2, 2, 2), (258, 34, 130)])
def test_cuda_gemm_fp64_tensor_path(m, k, n):
    """Even shapes take the DMMA path (gemm_mma.cu); ragged tiles included."""
    rng = np.random.default_rng(m + k + n)
    a = rng.standard_normal((m, k))
    b = rng.standard_normal((k, n))
    got = api.cuda_gemm(a, b, precision=64)
    assert O.rel_err(got, a @ b) < 1e-14


def test_cuda_gemm():
    rng = np.random.default_rng(3)
    a = rng.standard_normal((130, 77))
    b = rng.standard_normal((77, 211))
    for prec in (64, 32):
        got = api.cuda_gemm(a, b, precision=prec)
        want = a.astype(np.float32 if prec == 32 else np.float64).astype(np.float64) @ \
            b.astype(np.float32 if prec == 32 else np.float64).astype(np.float64)
        assert O.rel_err(got, want) < (1e-13 if prec == 64 else 1e-7)


def test_errors_and_paths():
    x, y = W.latent_regression(50, 20, 2, 2, 0.5, 9, dtype=np.float64)
    with pytest.raises(api._lib.FastplsError, match="invalid resident SIMPLS dimensions"):
        api.fit_resident(x, y, ncomp=60)
    model = api.fit_resident(x, y, ncomp=3)
    with pytest.raises(api._lib.FastplsError, match="strictly increasing"):
        model.predict_path(x, [2, 1])
    with pytest.raises(api._lib.FastplsError, match="LDA requires class labels"):
        model.predict_path(x, [1], lda=True)
    err, cap = api._lib.error_buffer()
    bad = np.zeros(5)
    rc = api._lib.load().fastpls_resident_export(
        api.C.c_void_p(model.handle), 0, bad.ctypes.data_as(api.C.c_void_p), 5, err, cap)
    assert rc == 1 and b"invalid resident field output size" in err.value
    model.close()
