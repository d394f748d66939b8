"""The numpy oracle against the compiled reference core on fresh seeded
inputs (runs where oracle/_ref was built from the reference sources)."""
import numpy as np
import pytest

from fastpls_b200 import workloads as W
from oracle import pls_oracle as O
from oracle import ref

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("shape", [(50, 200, 2), (200, 40, 5)])
def test_simpls(seed, shape):
    n, p, m = shape
    x, y = W.latent_regression(n, p, m, 3, 0.4, seed, dtype=np.float64)
    a = O.simpls_fit(x, y, ncomp=6, scaling=1)
    b = ref.simpls_fit(x, y, ncomp=6, scaling=1)
    assert O.rel_err(a["R"] @ a["Q"].T, b["R"] @ b["Q"].T) < 1e-8
    assert O.rel_err(O.align_signs(a["T"], b["T"]), b["T"]) < 1e-8


def test_cv_regression_uneven_folds():
    x, y = W.latent_regression(150, 70, 3, 3, 0.4, 9, dtype=np.float64)
    folds = W.uneven_folds(150, 6, 9)
    a = O.cv_regression(x, y, folds, [1, 2, 4], scaling=2)
    b = ref.cv_regression(x, y, folds, [1, 2, 4], scaling=2)
    assert np.allclose(a["q2"], b["q2"], rtol=1e-9)


def test_cv_fold_zero_rows_always_train():
    # fold id 0 = never held out (cross_validation.hpp:772-798)
    x, y = W.latent_regression(90, 30, 2, 3, 0.4, 10, dtype=np.float64)
    folds = W.uneven_folds(90, 3, 10)
    folds[:7] = 0
    a = O.cv_regression(x, y, folds, [1, 3], scaling=1, store_predictions=True)
    b = ref.cv_regression(x, y, folds, [1, 3], scaling=1, store_predictions=True)
    assert np.allclose(a["rmsd"], b["rmsd"], rtol=1e-9)
