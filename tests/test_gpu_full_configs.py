"""The PLS-SVD + LDA classification configuration at full size.

20000 x 50000 FP32 predictors from a latent model with k = 20 factors whose
scales decay as 100 * 0.8^i, noise sd 0.1, column-centred; 10 classes from
argmax(T C), C ~ N(0, 1) 20 x 10; PLS-SVD with ncomp 20 capped at
classes - 1 = 9 (src/cuda_resident_plssvd.cuh:89-91; the R layer caps
ncomp, R/main.R:192); LDA on the scores. Checked against FP64 host
computations on the same inputs: the weights against the leading left
singular vectors of the centred label cross-product, and the LDA labels of
2000 rows against the oracle's LDA trained on host-computed scores."""
import numpy as np
import pytest

from fastpls_b200 import api
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu


def test_plssvd_lda_full_size():
    torch = pytest.importorskip("torch")
    n, p, k, classes, a = 20_000, 50_000, 20, 10, 9
    dev = torch.device("cuda")
    g = torch.Generator(device=dev).manual_seed(2)
    sigma = 100.0 * 0.8 ** torch.arange(k, device=dev, dtype=torch.float32)
    t = torch.randn(n, k, generator=g, device=dev) * sigma
    w = torch.randn(p, k, generator=g, device=dev)
    c = torch.randn(k, classes, generator=g, device=dev)
    xt = w @ t.T                                   # p x n = column-major n x p
    xt += 0.1 * torch.randn(p, n, generator=g, device=dev)
    xt -= xt.mean(dim=1, keepdim=True)
    lab = (torch.argmax(t @ c, dim=1) + 1).to(torch.int32).cpu().numpy()
    x = xt.cpu().numpy().T                          # n x p, Fortran order
    del xt, t, w
    torch.cuda.empty_cache()
    assert x.flags.f_contiguous
    assert np.bincount(lab, minlength=classes + 1)[1:].min() > 0

    model = api.fit_resident(x, labels=lab, classes=classes, ncomp=a, method="plssvd",
                             precision=32, oversample=10, power=2)
    R = model.export(0).astype(np.float64)
    probe = x[::10]
    pre = [1, 3, 5, 9]
    got = model.classify_path(probe, pre, lda=True)
    model.close()

    # host FP64: column means, centred label cross-product, scores
    mu = np.zeros(p)
    for r0 in range(0, n, 2000):
        mu += x[r0:r0 + 2000].astype(np.float64).sum(axis=0)
    mu /= n
    onehot = np.zeros((n, classes))
    onehot[np.arange(n), lab - 1] = 1.0
    yc = onehot - onehot.mean(axis=0)
    s = np.zeros((p, classes))
    for r0 in range(0, n, 2000):
        s += (x[r0:r0 + 2000].astype(np.float64) - mu).T @ yc[r0:r0 + 2000]
    u = np.linalg.svd(s, full_matrices=False)[0][:, :a]
    assert O.rel_err(O.align_signs(R, u), u) < 1e-5

    u = O.align_signs(u, R)
    T = np.zeros((n, a))
    for r0 in range(0, n, 2000):
        T[r0:r0 + 2000] = (x[r0:r0 + 2000].astype(np.float64) - mu) @ u
    lda = O.lda_train(T, lab, classes, pre)
    tp = T[::10]
    for j in range(len(pre)):
        want = O.row_argmax(O.lda_discriminants(lda[j], tp[:, :pre[j]]))
        assert np.array_equal(got[j][:, 0], want)
