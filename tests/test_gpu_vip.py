"""Variable importance in projection on the device (fastpls_b200_resident_vip)
against the oracle restatement of vip_values (src/r_api.cpp:3973-4025)."""
import numpy as np
import pytest

from fastpls_b200 import api, workloads as W
from fastpls_b200._lib import FastplsError
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu


def _close(a, b, tol):
    assert a.shape == b.shape
    assert np.array_equal(np.isnan(a), np.isnan(b))
    ok = ~np.isnan(b)
    assert O.rel_err(a[ok], b[ok]) < tol


@pytest.mark.parametrize("method", ["simpls", "plssvd", "opls"])
def test_vip_matches_oracle(method):
    x, y = W.latent_regression(260, 140, 3, 4, 0.4, 91, dtype=np.float64)
    kw = {"north": 1} if method == "opls" else {}
    model = api.fit_resident(x, y, ncomp=3, method=method, **kw)
    got = model.vip()
    want = O.vip(model.export(0), model.export(1), model.export(2))
    _close(got, want, 1e-12)
    if method == "simpls":
        ref = O.simpls_fit(x, y, ncomp=3)
        _close(got, O.vip(ref["R"], ref["Q"], ref["T"]), 1e-9)
    model.close()


def test_vip_kernel_pls_and_single_response():
    x, y = W.latent_regression(120, 30, 1, 3, 0.4, 92, dtype=np.float64)
    model = api.fit_resident(x, y, ncomp=4, method="kernelpls", gamma=0.01)
    got = model.vip()
    assert got.shape == (1, 4, 120)
    _close(got, O.vip(model.export(0), model.export(1), model.export(2)), 1e-12)
    model.close()


def test_vip_needs_training_scores():
    x, y = W.latent_regression(100, 20, 2, 3, 0.4, 93, dtype=np.float64)
    model = api.fit_resident(x, y, ncomp=2)
    bare = api.import_model(api.export_model(model, scores=False))
    with pytest.raises(FastplsError, match="fit = TRUE"):
        bare.vip()
    model.close()
    bare.close()
