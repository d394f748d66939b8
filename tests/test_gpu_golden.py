"""Device results against the golden fixtures written by the compiled
reference core (tests/golden/*.npz, made by tests/golden/make_golden.py from
oracle/_ref, i.e. fastPLS inst/include/fastpls/core in FP64): the GPU path is
compared with the reference's own outputs directly, without the numpy
oracle in between. FP64 storage; tolerances as the reference's own
GPU-vs-CPU pins (1e-10 for OPLS / kernel PLS predictions,
tests/testthat/test-cuda-resident-public.R:162) or 1e-9 on coefficients and
scores after sign alignment; class predictions and accuracies exact."""
import os

import numpy as np
import pytest

from fastpls_b200 import api
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


def _aligned(got, want):
    return O.rel_err(O.align_signs(got, want), want)


@pytest.mark.parametrize("scaling", [1, 2, 3])
def test_simpls_regression_vs_reference(scaling):
    g = gold(f"simpls_reg_s{scaling}")
    m = api.fit_resident(g["x"], g["y"], ncomp=8, scaling=scaling, precision=64)
    R, Q, T = m.export(0), m.export(1), m.export(2)
    sg = np.where(np.einsum("ij,ij->j", R, g["R"]) < 0, -1.0, 1.0)
    assert O.rel_err(R * sg, g["R"]) < 1e-9
    assert O.rel_err(Q * sg, g["Q"]) < 1e-9
    assert O.rel_err(T * sg, g["T"]) < 1e-9
    # the fixture's X is column-centred already: its means are rounding
    # noise, compared in absolute terms against the scale of X
    xs = np.abs(g["x"]).max()
    assert np.abs(m.export(3) - g["centre"]).max() < 1e-13 * xs
    assert O.rel_err(m.export(4), g["scale"]) < 1e-12
    assert O.rel_err(m.export(5), g["ymean"]) < 1e-12
    m.close()


def test_simpls_classification_vs_reference():
    g = gold("simpls_cls")
    m = api.fit_resident(g["x"], labels=g["labels"], classes=4, ncomp=5, scaling=2,
                         precision=64)
    assert _aligned(m.export(0), g["R"]) < 1e-9
    assert _aligned(m.export(2), g["T"]) < 1e-9
    assert O.rel_err(m.export(5), g["ymean"]) < 1e-12
    m.close()


def test_plssvd_vs_reference():
    g = gold("plssvd_reg")
    m = api.fit_resident(g["x"], g["y"], ncomp=3, method="plssvd", precision=64)
    assert _aligned(m.export(0), g["R"]) < 1e-9
    assert _aligned(m.export(2), g["T"]) < 1e-9
    m.close()


@pytest.mark.parametrize("family", ["simpls", "plssvd"])
def test_cv_regression_vs_reference(family):
    g = gold(f"cv_reg_{family}")
    pre = [int(v) for v in g["prefixes"]]
    got = api.cv_regression(g["x"], g["y"], g["folds"], pre, method=family, precision=64,
                            store_predictions=True)
    for key, gk in (("q2", "q2"), ("rmsd", "rmsd"), ("observed_r2", "r2")):
        assert np.allclose(got[key], g[gk], rtol=1e-9, atol=1e-12), key
    assert O.rel_err(np.asarray(got["predictions"]), g["predictions"]) < 1e-9


@pytest.mark.parametrize("head", [0, 1])
def test_cv_classification_vs_reference(head):
    g = gold(f"cv_cls_h{head}")
    pre = [int(v) for v in g["prefixes"]]
    got = api.cv_classification(g["x"], g["labels"], 4, g["folds"], pre, lda=bool(head),
                                precision=64, store_predictions=True)
    assert np.array_equal(got["metrics"], g["metrics"])
    assert np.array_equal(np.asarray(got["predictions"]), g["predictions"])


@pytest.mark.parametrize("north", [1, 2])
def test_opls_vs_reference(north):
    g = gold(f"opls_n{north}")
    m = api.fit_resident(g["x"], g["y"], ncomp=4, scaling=2, method="opls", north=north,
                         precision=64)
    pred = m.predict_path(g["xtest"], [4])[0]
    assert O.rel_err(pred, g["pred"]) < 1e-10
    m.close()


@pytest.mark.parametrize("kind", [2, 3])
def test_kernelpls_vs_reference(kind):
    g = gold(f"kernelpls_k{kind}")
    m = api.fit_resident(g["x"], g["y"], ncomp=5, scaling=1, method="kernelpls",
                         kernel={2: "rbf", 3: "poly"}[kind], gamma=float(g["gamma"]),
                         degree=int(g["degree"]), coef0=1.0, precision=64)
    pred = m.predict_path(g["xtest"], [5])[0]
    assert O.rel_err(pred, g["pred"]) < 1e-10
    m.close()
