"""One-pass projection X R for 3..16 columns of a large X (bulk-copy stages
carrying their rows of R): predictions at those widths against the oracle,
and BF16 storage against FP32 storage of the same values bit for bit (the
partition and every sum's order depend on n and p only)."""
import numpy as np
import pytest
import torch

from fastpls_b200 import api, workloads as W
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ncomp", [3, 9, 16])
def test_wide_projection_matches_oracle(ncomp):
    n, p, q = 2049, 9000, 3          # 18.4 M elements: the one-pass form; ragged last row block
    x, y = W.latent_regression(n, p, q, 6, 0.4, 60 + ncomp, dtype=np.float32)
    model = api.fit_resident(x, y, ncomp=ncomp, precision=32)
    pre = sorted({1, max(1, ncomp // 2), ncomp})
    got = model.predict_path(x, pre)
    model.close()
    ref = O.simpls_fit(x.astype(np.float64), y.astype(np.float64), ncomp=ncomp)
    for j, k in enumerate(pre):
        err = O.rel_err(got[j].astype(np.float64), O.simpls_predict(ref, x.astype(np.float64), k))
        assert err < 1e-5, (k, err)


def test_wide_projection_bf16_equals_fp32_storage():
    n, p, q, a = 2049, 9000, 2, 9
    xf, y = W.latent_regression(n, p, q, 6, 0.4, 77, dtype=np.float32)
    xb = torch.from_numpy(np.ascontiguousarray(xf.T)).to(torch.bfloat16)   # p x n, row-major
    x16 = xb.float().numpy().T                                            # the BF16 values as FP32
    bits = xb.view(torch.int16).numpy().view(np.uint16).T                 # n x p, F-order
    m16 = api.fit_resident(bits, y, ncomp=a, precision=16)
    m32 = api.fit_resident(np.asfortranarray(x16), y, ncomp=a, precision=32)
    # the whole matrix again: large enough for the one-pass form
    assert np.array_equal(m16.predict_path(bits, [1, a]),
                          m32.predict_path(np.asfortranarray(x16), [1, a]))
    m16.close()
    m32.close()
