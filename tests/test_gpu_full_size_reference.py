"""The full-size configurations against the compiled FP64 reference core.

* Mixed precision: X 100000 x 20000 stored in BF16 (column scales
  log-normal), 10 responses, 50 SIMPLS components. The reference
  (fit_simpls_preprocessed<double>, inst/include/fastpls/core/simpls.hpp:
  479-763) runs in FP64 on the host on the same BF16-rounded values. R, Q, T
  (after per-component sign alignment), B = R Q^T and the predictions of 4000
  rows at prefixes 1, 10, 25 and 50 must agree within 1e-5 relative.
* PLS-SVD + LDA: X 20000 x 50000 FP32, 10 classes, ncomp capped at
  classes - 1 = 9 (src/cuda_resident_plssvd.cuh:89-91). The reference
  PLS-SVD (plssvd.hpp:57-166) and its LDA (lda.hpp:156-223) on the
  reference's own scores give the labels of 2000 rows at prefixes 1, 3, 5
  and 9; the device labels must be identical.

Each test prints its error report (run with -s to see it)."""
import os

import numpy as np
import pytest

from fastpls_b200 import api
from fastpls_b200 import workloads as W
from oracle import pls_oracle as O
from oracle import ref as R_

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not R_.available(),
                               reason="compiled reference core (oracle/_ref) not built")


def _align(R, Rref):
    """Signs that align each column of R with the matching reference column."""
    return np.where(np.einsum("ij,ij->j", R, Rref) < 0.0, -1.0, 1.0)


def _prefix_predictions(ref, xp, prefixes):
    T = (xp - ref["centre"]) / ref["scale"] @ ref["R"]
    return [ref["ymean"] + T[:, :k] @ ref["Q"][:, :k].T for k in prefixes]


@needs_ref
def test_bf16_mixed_precision_full_size_vs_reference():
    n, p, m, a = 100_000, 20_000, 10, 50
    bits, y = W.mixed_precision_config(seed=4, n=n, p=p, m=m, k=50)
    rows = np.arange(0, n, 25)[:4000]
    pre = [1, 10, 25, 50]
    model = api.fit_resident(bits, y, ncomp=a, precision=16)
    got_pred = model.predict_path(bits[rows], pre).astype(np.float64)
    R = model.export(0).astype(np.float64)
    Q = model.export(1).astype(np.float64)
    T = model.export(2).astype(np.float64)
    model.close()

    x64 = W.bf16_to_f64(bits)
    del bits
    R_.set_threads(os.cpu_count() or 1)
    ref = R_.simpls_fit(x64, y.astype(np.float64), ncomp=a, scaling=1)
    want_pred = _prefix_predictions(ref, x64[rows], pre)
    del x64
    assert ref["R"].shape[1] == a

    sg = _align(R, ref["R"])
    report = {
        "R": O.rel_err(R * sg, ref["R"]),
        "Q": O.rel_err(Q * sg, ref["Q"]),
        "T": O.rel_err(T * sg, ref["T"]),
    }
    for k in pre:
        report[f"B[{k}]"] = O.rel_err(R[:, :k] @ Q[:, :k].T, ref["R"][:, :k] @ ref["Q"][:, :k].T)
    for j, k in enumerate(pre):
        report[f"Yhat[{k}]"] = O.rel_err(got_pred[j], want_pred[j])
    print("\nmixed precision 100000 x 20000 BF16, 50 components, rel err vs FP64 reference:",
          {k: f"{v:.2e}" for k, v in report.items()},
          f"reference fit {ref['seconds']:.1f} s")
    for key, err in report.items():
        assert err < 1e-5, (key, err)


@needs_ref
def test_plssvd_lda_full_size_vs_reference():
    n, p, classes, a = 20_000, 50_000, 10, 9
    x, lab = W.plssvd_lda_config(seed=2, n=n, p=p, k=20, classes=classes)
    pre = [1, 3, 5, 9]
    probe = np.arange(0, n, 10)
    model = api.fit_resident(x, labels=lab, classes=classes, ncomp=a, method="plssvd",
                             precision=32, oversample=10, power=2)
    got = model.classify_path(x[probe], pre, lda=True)
    Rg = model.export(0).astype(np.float64)
    model.close()

    x64 = np.asfortranarray(x, dtype=np.float64)
    del x
    R_.set_threads(os.cpu_count() or 1)
    ref = R_.plssvd_fit(x64, labels=lab, classes=classes, prefixes=pre, scaling=1,
                        oversample=10, power=2)
    tp = (x64[probe] - ref["centre"]) @ ref["R"]
    del x64
    _, want = R_.lda(ref["T"], lab, classes, pre, tp)
    err_r = O.rel_err(Rg * _align(Rg, ref["R"]), ref["R"])
    flips = [int(np.sum(got[j][:, 0] != want[:, j])) for j in range(len(pre))]
    print(f"\nPLS-SVD + LDA 20000 x 50000 FP32: R rel err {err_r:.2e}, "
          f"label differences per prefix {flips} of {len(probe)} rows")
    assert err_r < 1e-5
    for j in range(len(pre)):
        assert np.array_equal(got[j][:, 0], want[:, j]), (pre[j], flips[j])
