"""Predictors stored in BF16 (precision 16) through the C ABI.

The mixed-precision configuration (100000 x 20000 predictors in BF16, latent
k = 50 with log-normal column scales, 10 responses, ncomp = 50) keeps X in
BF16 on the device; every product is widened to FP64, so the fit equals the
FP64 fit of the BF16-rounded values. Checked here: against the FP64 oracle on
the same rounded values at a reduced size, bit-equality with FP32 storage of
the same values, and at the full size the first direction against a chunked
FP64 cross-product on the host, orthonormal scores and storage equality."""
import numpy as np
import pytest

from fastpls_b200 import api, workloads as W
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu

TOL32 = 1e-6   # results come back in FP32


def _data(n, p, m, k, seed):
    x, y = W.latent_regression(n, p, m, k, 0.5, seed, log_normal_scales=True,
                               dtype=np.float32)
    bits = api.to_bf16(x)
    return bits, api.from_bf16(bits).astype(np.float64).reshape(x.shape), y


def test_simpls_bf16_vs_oracle():
    bits, xv, y = _data(3000, 1500, 10, 50, 71)
    tb, tv, _ = _data(400, 1500, 10, 50, 72)
    model = api.fit_resident(bits, y, ncomp=50, precision=16)
    ref = O.simpls_fit(xv, y.astype(np.float64), ncomp=50, scaling=1)
    pre = [1, 10, 25, 50]
    pred = model.predict_path(tb, pre)
    assert pred.dtype == np.float32
    for j, k in enumerate(pre):
        assert O.rel_err(pred[j].astype(np.float64), O.simpls_predict(ref, tv, k)) < TOL32
    sc = model.project(tb, 50).astype(np.float64)
    want = O.simpls_project(ref, tv, 50)
    assert O.rel_err(O.align_signs(sc, want), want) < TOL32
    R = model.export(0).astype(np.float64)
    assert O.rel_err(O.align_signs(R, ref["R"]), ref["R"]) < TOL32
    model.close()


@pytest.mark.parametrize("scaling", [1, 2])
def test_bf16_equals_fp32_storage(scaling):
    bits, xv, y = _data(2500, 900, 4, 12, 73)
    tb, tv, _ = _data(300, 900, 4, 12, 74)
    m16 = api.fit_resident(bits, y, ncomp=12, precision=16, scaling=scaling)
    m32 = api.fit_resident(xv.astype(np.float32), y, ncomp=12, precision=32, scaling=scaling)
    pre = [1, 6, 12]
    assert np.array_equal(m16.predict_path(tb, pre),
                          m32.predict_path(tv.astype(np.float32), pre))
    for f in range(8):
        assert np.array_equal(m16.export(f), m32.export(f))
    m16.close()
    m32.close()


def test_plssvd_opls_kernelpls_bf16():
    bits, xv, y = _data(600, 300, 3, 8, 75)
    tb, tv, _ = _data(100, 300, 3, 8, 76)
    yd = y.astype(np.float64)
    m = api.fit_resident(bits, y, ncomp=3, method="plssvd", precision=16)
    ref = O.plssvd_fit(xv, yd, prefixes=[1, 2, 3])
    pred = m.predict_path(tb, [1, 2, 3])
    for j in range(3):
        assert O.rel_err(pred[j].astype(np.float64), O.plssvd_predict(ref, tv, j)) < TOL32
    m.close()
    m = api.fit_resident(bits, y, ncomp=4, method="opls", north=1, precision=16)
    ref = O.opls_fit(xv, yd, ncomp=4, north=1)
    pred = m.predict_path(tb, [2, 4])
    for j, k in enumerate([2, 4]):
        assert O.rel_err(pred[j].astype(np.float64), O.opls_predict(ref, tv, k)) < TOL32
    m.close()
    m = api.fit_resident(bits, y, ncomp=5, method="kernelpls", kernel="rbf",
                         gamma=2e-5, precision=16)
    ref = O.kernelpls_fit(xv, yd, ncomp=5, kind=2, gamma=2e-5)
    pred = m.predict_path(tb, [5])
    assert O.rel_err(pred[0].astype(np.float64), O.kernelpls_predict(ref, tv, 5)) < TOL32
    m.close()


def test_bf16_classification_lda():
    x, lab = W.latent_classification(800, 400, 5, 4, 0.5, 77, dtype=np.float32)
    xt, _ = W.latent_classification(200, 400, 5, 4, 0.5, 78, dtype=np.float32)
    bits, tb = api.to_bf16(x), api.to_bf16(xt)
    xv = api.from_bf16(bits).astype(np.float64).reshape(x.shape)
    tv = api.from_bf16(tb).astype(np.float64).reshape(xt.shape)
    model = api.fit_resident(bits, labels=lab, classes=5, ncomp=6, precision=16)
    ref = O.simpls_fit(xv, labels=lab, classes=5, ncomp=6)
    pre = [2, 6]
    got = model.classify_path(tb, pre, lda=True)
    lda = O.lda_train(ref["T"], lab, 5, pre)
    tt = O.simpls_project(ref, tv, 6)
    for j in range(len(pre)):
        assert np.array_equal(got[j][:, 0], O.row_argmax(O.lda_discriminants(lda[j], tt)))
    model.close()


def test_full_size_bf16_configuration():
    """100000 x 20000 BF16 predictors, 10 responses, 50 components."""
    torch = pytest.importorskip("torch")
    n, p, m, k, a = 100_000, 20_000, 10, 50, 50
    g = torch.Generator(device="cuda").manual_seed(4)
    dev = torch.device("cuda")
    t = torch.randn(n, k, generator=g, device=dev)
    w = torch.randn(p, k, generator=g, device=dev)
    scale = torch.exp(torch.randn(p, generator=g, device=dev))
    c = torch.randn(k, m, generator=g, device=dev)
    # column-major n x p == row-major p x n
    xt = (w * scale[:, None]) @ t.T
    xt += 0.5 * torch.randn(p, n, generator=g, device=dev)
    xt -= xt.mean(dim=1, keepdim=True)
    xb = xt.to(torch.bfloat16)
    del xt
    y = (t @ c + 0.1 * torch.randn(n, m, generator=g, device=dev)).T.contiguous()
    bits = xb.view(torch.int16).cpu().numpy().view(np.uint16).T      # n x p, F-order
    x32 = xb.float().cpu().numpy().T                                  # same values, FP32
    yh = y.cpu().numpy().T
    del xb, t, w, y
    torch.cuda.empty_cache()
    assert bits.flags.f_contiguous and x32.flags.f_contiguous

    m16 = api.fit_resident(bits, yh, ncomp=a, precision=16)
    rows = np.arange(0, n, 25)[:4000]
    probe16 = bits[rows]
    probe32 = x32[rows]
    p16 = m16.predict_path(probe16, [1, 10, 50])
    R = m16.export(0).astype(np.float64)
    T = m16.export(2).astype(np.float64)
    m16.close()

    m32 = api.fit_resident(x32, yh, ncomp=a, precision=32)
    assert np.array_equal(p16, m32.predict_path(probe32, [1, 10, 50]))
    assert np.array_equal(R, m32.export(0).astype(np.float64))
    m32.close()

    # scores are orthonormal
    G = T.T @ T
    assert np.abs(G - np.eye(a)).max() < 1e-4
    # first direction = dominant left singular vector of S = Xc^T Yc (FP64 host)
    yc = yh.astype(np.float64) - yh.astype(np.float64).mean(axis=0)
    s = np.zeros((p, m))
    colsum = np.zeros(p)
    for r0 in range(0, n, 5000):
        blk = x32[r0:r0 + 5000].astype(np.float64)
        s += blk.T @ yc[r0:r0 + 5000]
        colsum += blk.sum(axis=0)
    s -= np.outer(colsum / n, yc.sum(axis=0))
    u = np.linalg.svd(s, full_matrices=False)[0][:, :1]
    r1 = R[:, :1] / np.linalg.norm(R[:, :1])
    assert O.rel_err(O.align_signs(r1, u), u) < 1e-5
