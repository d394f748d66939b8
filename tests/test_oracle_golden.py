"""The numpy oracle against the committed golden fixtures (outputs of the
reference core compiled from its own sources; see tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from oracle import pls_oracle as O

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(G, name + ".npz"))


@pytest.mark.parametrize("sc", [1, 2, 3])
def test_simpls_regression_golden(sc):
    f = load(f"simpls_reg_s{sc}")
    m = O.simpls_fit(f["x"], f["y"], ncomp=8, scaling=sc)
    for k in ("R", "T", "V"):
        assert O.rel_err(O.align_signs(m[k], f[k]), f[k]) < 1e-9, k
    assert O.rel_err(m["R"] @ m["Q"].T, f["R"] @ f["Q"].T) < 1e-9
    assert np.allclose(m["centre"], f["centre"]) and np.allclose(m["scale"], f["scale"])


def test_simpls_classification_golden():
    f = load("simpls_cls")
    m = O.simpls_fit(f["x"], labels=f["labels"], classes=4, ncomp=5, scaling=2)
    assert O.rel_err(O.align_signs(m["T"], f["T"]), f["T"]) < 1e-10
    assert np.allclose(m["ymean"], f["ymean"])


def test_plssvd_golden():
    f = load("plssvd_reg")
    m = O.plssvd_fit(f["x"], f["y"], prefixes=[1, 2, 3], scaling=1)
    assert np.allclose(m["sigma"], f["sigma"], rtol=1e-12)
    for j in range(3):
        a = m["T"][:, :j + 1] @ m["W"][j]
        b = f["T"][:, :j + 1] @ f[f"W{j + 1}"]
        assert O.rel_err(a, b) < 1e-12


@pytest.mark.parametrize("name,fam", [("simpls", 3), ("plssvd", 1)])
def test_cv_regression_golden(name, fam):
    f = load(f"cv_reg_{name}")
    out = O.cv_regression(f["x"], f["y"], f["folds"], f["prefixes"], scaling=1,
                          family=fam, store_predictions=True)
    assert np.allclose(out["q2"], f["q2"], rtol=1e-10)
    assert np.allclose(out["rmsd"], f["rmsd"], rtol=1e-10)
    assert np.allclose(out["observed_r2"], f["r2"], rtol=1e-10)
    assert O.rel_err(out["predictions"], f["predictions"]) < 1e-10


@pytest.mark.parametrize("head", [0, 1])
def test_cv_classification_golden(head):
    f = load(f"cv_cls_h{head}")
    out = O.cv_classification(f["x"], f["labels"], 4, f["folds"], f["prefixes"],
                              scaling=1, family=3, head=head,
                              store_predictions=True)
    assert np.array_equal(out["predictions"], f["predictions"])
    assert np.allclose(out["metrics"], f["metrics"])


def test_lda_golden():
    f = load("lda")
    pre = [int(v) for v in f["prefixes"]]
    models = O.lda_train(f["train"], f["labels"], 3, pre)
    for j in range(len(pre)):
        d = O.lda_discriminants(models[j], f["test"])
        assert O.rel_err(d, f["disc"][j]) < 1e-12
        assert np.array_equal(O.row_argmax(d), f["pred"][:, j])


@pytest.mark.parametrize("north", [1, 2])
def test_opls_golden(north):
    f = load(f"opls_n{north}")
    m = O.opls_fit(f["x"], f["y"], ncomp=4, scaling=2, north=north)
    assert O.rel_err(O.opls_predict(m, f["xtest"], 4), f["pred"]) < 1e-9


@pytest.mark.parametrize("kind", [2, 3])
def test_kernelpls_golden(kind):
    f = load(f"kernelpls_k{kind}")
    m = O.kernelpls_fit(f["x"], f["y"], ncomp=5, scaling=1, kind=kind,
                        gamma=float(f["gamma"]), degree=int(f["degree"]), coef0=1.0)
    assert O.rel_err(O.kernelpls_predict(m, f["xtest"], 5), f["pred"]) < 1e-10
