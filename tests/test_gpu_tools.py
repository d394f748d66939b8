"""fastcor and fastsvd on the device vs the oracle / exact numpy SVD."""
import numpy as np
import pytest

from fastpls_b200 import api, workloads as W
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("byrow", [True, False])
def test_fastcor_matches_oracle(byrow):
    rng = np.random.default_rng(11)
    a = rng.standard_normal((64, 90))
    b = rng.standard_normal((64, 90))
    a[3] = 1.0          # zero spread unit (byrow) -> NaN row/column
    got = api.fastcor(a, byrow=byrow)
    want = O.fastcor(a, byrow=byrow)
    assert np.array_equal(np.isnan(got), np.isnan(want))
    m = ~np.isnan(want)
    assert np.max(np.abs(got[m] - want[m])) < 1e-13
    got_ab = api.fastcor(a, b, byrow=byrow, diag=False)
    assert np.nanmax(np.abs(got_ab - O.fastcor(a, b, byrow=byrow, diag=False))) < 1e-13
    got_d = api.fastcor(a, b, byrow=byrow, diag=True)
    assert np.nanmax(np.abs(got_d - O.fastcor(a, b, byrow=byrow, diag=True))) < 1e-13
    if not byrow:
        assert np.allclose(got, np.corrcoef(a.T), equal_nan=True)


@pytest.mark.parametrize("precision", [64, 32])
def test_fastsvd_matches_exact_truncated_svd(precision):
    x, _ = W.latent_regression(300, 220, 1, 8, 0.05, 61, dtype=np.float64)
    if precision == 32:
        x = x.astype(np.float32)
    x64 = x.astype(np.float64)
    k = 6
    u, d, v = api.fastsvd(x, k, oversample=20, power=4, seed=7, precision=precision)
    U, S, Vt = np.linalg.svd(x64, full_matrices=False)
    assert np.allclose(d, S[:k], rtol=1e-9)
    assert O.rel_err(O.align_signs(u, U[:, :k]), U[:, :k]) < 1e-7
    assert O.rel_err(O.align_signs(v, Vt[:k].T), Vt[:k].T) < 1e-7
    assert O.rel_err((u * d) @ v.T, (U[:, :k] * S[:k]) @ Vt[:k]) < 1e-9


def test_fastsvd_full_span_is_exact():
    rng = np.random.default_rng(5)
    x = rng.standard_normal((40, 12))
    u, d, v = api.fastsvd(x, 5, oversample=32, power=0, seed=1)
    S = np.linalg.svd(x, compute_uv=False)
    assert np.allclose(d, S[:5], rtol=1e-11)
