"""The persistent single-fit SIMPLS launch (csrc/persistent.cu) against the
per-kernel component loop and the FP64 oracle: same model to rounding, on
FP64, FP32 and BF16 storage, for odd shapes (rows not a multiple of the
vector width, columns not a multiple of the tile width, more CTAs than
columns), regression and classification, and over several response counts.

The two device paths sum in different orders; late components that fit
noise amplify that to a few 1e-10, hence 1e-8 between them. Against the
oracle (a direct SVD of S where the device, like the reference, solves the
m x m right Gram) the many-response case with small eigen-gaps in its late
components agrees to ~2e-8 on B; the contract is 1e-5."""
import numpy as np
import pytest

from fastpls_b200 import api
from fastpls_b200 import workloads as W
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu


def _fit_both(x, y=None, labels=None, classes=None, ncomp=5, precision=64, scaling="centering"):
    out = []
    old = api.persistent()
    try:
        for on in (True, False):
            api.set_persistent(on)
            m = api.fit_resident(x, y, labels=labels, classes=classes, ncomp=ncomp,
                                 precision=precision, scaling=scaling)
            out.append({f: m.export(f).astype(np.float64) for f in (0, 1, 2, 6)})
            m.close()
    finally:
        api.set_persistent(old)
    return out


@pytest.mark.parametrize("n,p,m,a", [(301, 517, 3, 8), (1000, 37, 2, 6), (4097, 2050, 10, 12),
                                     (64, 9000, 1, 5), (2500, 3001, 32, 7)])
def test_persistent_matches_kernel_loop_and_oracle(n, p, m, a):
    x, y = W.latent_regression(n, p, m, 6, 0.4, n + p, dtype=np.float64)
    got, loop = _fit_both(x, y, ncomp=a)
    for f in (0, 1, 2, 6):
        assert O.rel_err(got[f], loop[f]) < 1e-8, f
    ref = O.simpls_fit(x, y, ncomp=a)
    assert O.rel_err(O.align_signs(got[0], ref["R"]), ref["R"]) < 1e-8
    B = got[0] @ got[1].T
    assert O.rel_err(B, ref["R"] @ ref["Q"].T) < 1e-7


@pytest.mark.parametrize("scaling", ["centering", "autoscaling", "none"])
def test_persistent_scalings(scaling):
    x, y = W.latent_regression(700, 900, 3, 5, 0.5, 9, dtype=np.float32)
    got, loop = _fit_both(x, y, ncomp=9, precision=32, scaling=scaling)
    for f in (0, 1, 2):
        assert O.rel_err(got[f], loop[f]) < 1e-8, f


def test_persistent_classification():
    x, lab = W.latent_classification(900, 700, 6, 4, 0.5, 17, dtype=np.float32)
    got, loop = _fit_both(x, labels=lab, classes=6, ncomp=8, precision=32)
    for f in (0, 1, 2):
        assert O.rel_err(got[f], loop[f]) < 1e-8, f


def test_persistent_bf16_equals_fp32_storage():
    torch = pytest.importorskip("torch")
    x, y = W.latent_regression(3001, 1999, 4, 6, 0.5, 23, dtype=np.float32)
    xb = torch.from_numpy(np.ascontiguousarray(x.T)).to(torch.bfloat16)
    bits = xb.view(torch.int16).numpy().view(np.uint16).T          # n x p, F-order
    x32 = np.asfortranarray(xb.float().numpy().T)
    m16 = api.fit_resident(bits, y, ncomp=10, precision=16)
    m32 = api.fit_resident(x32, y, ncomp=10, precision=32)
    for f in (0, 1, 2):
        assert np.array_equal(m16.export(f), m32.export(f)), f
    m16.close()
    m32.close()
