"""Generate the golden fixtures in this directory from the compiled reference.

Run in a container that has the reference tree (for oracle/_ref):
    make -C oracle && python tests/golden/make_golden.py
Each fixture stores seeded inputs and the reference core's FP64 outputs
(oracle/_ref/libfastpls_ref.so = fastPLS inst/include/fastpls/core compiled
with the project's OpenBLAS adapter). The tests compare the numpy oracle and
the CUDA library against these files; they need neither the reference tree
nor the compiled harness.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from fastpls_b200 import workloads as W  # noqa: E402
from oracle import ref  # noqa: E402


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)


def main():
    ref.set_threads(1)
    # SIMPLS regression, three scalings (plain-SIMPLS shape, reduced)
    x, y = W.latent_regression(80, 60, 3, 4, 0.5, 101, dtype=np.float64)
    for sc in (1, 2, 3):
        m = ref.simpls_fit(x, y, ncomp=8, scaling=sc)
        save(f"simpls_reg_s{sc}", x=x, y=y, R=m["R"], Q=m["Q"], V=m["V"],
             T=m["T"], centre=m["centre"], scale=m["scale"], ymean=m["ymean"])
    # SIMPLS classification
    xc, lab = W.latent_classification(90, 40, 4, 3, 0.5, 102, dtype=np.float64)
    m = ref.simpls_fit(xc, labels=lab, classes=4, ncomp=5, scaling=2)
    save("simpls_cls", x=xc, labels=lab, R=m["R"], Q=m["Q"], T=m["T"],
         ymean=m["ymean"])
    # PLS-SVD regression with a prefix path
    m = ref.plssvd_fit(x, y, prefixes=[1, 2, 3], scaling=1)
    save("plssvd_reg", x=x, y=y, R=m["R"], T=m["T"], sigma=m["sigma"],
         W1=m["W"][0], W2=m["W"][1], W3=m["W"][2], ymean=m["ymean"])
    # regression CV (SIMPLS and PLS-SVD) on uneven folds
    folds = W.uneven_folds(80, 5, 103)
    for fam, name in ((3, "simpls"), (1, "plssvd")):
        pre = [1, 2, 3, 5, 8] if fam == 3 else [1, 2, 3]
        out = ref.cv_regression(x, y, folds, pre, scaling=1, family=fam,
                                store_predictions=True)
        save(f"cv_reg_{name}", x=x, y=y, folds=folds, prefixes=np.array(pre),
             q2=out["q2"], rmsd=out["rmsd"], r2=out["observed_r2"],
             predictions=out["predictions"])
    # classification CV with argmax and LDA heads
    f2 = W.uneven_folds(90, 4, 104)
    for head in (0, 1):
        out = ref.cv_classification(xc, lab, 4, f2, [1, 2, 3], scaling=1,
                                    family=3, head=head, store_predictions=True)
        save(f"cv_cls_h{head}", x=xc, labels=lab, folds=f2,
             prefixes=np.array([1, 2, 3]), metrics=out["metrics"],
             predictions=out["predictions"])
    # OPLS (exact filter) and kernel PLS predictions
    xt, _ = W.latent_regression(30, 60, 3, 4, 0.5, 106, dtype=np.float64)
    for north in (1, 2):
        pred = ref.opls_predict(x, y, 4, north, 2, xt)
        save(f"opls_n{north}", x=x, y=y, xtest=xt, pred=pred)
    for kind, gamma, degree in ((2, 0.02, 3), (3, 0.01, 2)):
        pred = ref.kernelpls_predict(x, y, 5, 1, kind, gamma, degree, 1.0, xt)
        save(f"kernelpls_k{kind}", x=x, y=y, xtest=xt, pred=pred,
             gamma=np.array(gamma), degree=np.array(degree))
    # LDA on scores
    ts = W.rng(105, 0).standard_normal((60, 4))
    lab3 = (np.arange(60) % 3 + 1).astype(np.int32)
    ts[:, 0] += lab3
    te = W.rng(105, 1).standard_normal((20, 4))
    disc, pred = ref.lda(ts, lab3, 3, [1, 2, 4], te)
    save("lda", train=ts, labels=lab3, test=te, prefixes=np.array([1, 2, 4]),
         disc=disc, pred=pred)


if __name__ == "__main__":
    main()
