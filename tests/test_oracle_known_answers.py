"""Pin the numpy oracle to the known answers of the reference's own C++ tests
(fastPLS core/tests/test_core_plssvd.cpp, test_core_simpls.cpp,
test_core_lda.cpp). The fixtures are restated from those files."""
import numpy as np

from oracle import pls_oracle as O


def _plssvd_fixture():
    # core/tests/test_core_plssvd.cpp:13-22
    v = np.arange(8) - 3.5
    x = np.stack([v, v * v - 5.25, np.where(np.arange(8) % 2 == 0, -1.0, 1.0)], 1)
    y = np.stack([2 * x[:, 0] - 0.5 * x[:, 1], x[:, 2] + 0.25 * x[:, 0]], 1)
    return x, y


def test_plssvd_known_answers():
    x, y = _plssvd_fixture()
    m = O.plssvd_fit(x, y, prefixes=[1, 2], scaling=3)
    pred = m["T"][:, :2] @ m["W"][1] + m["ymean"]
    error = float(((pred - y) ** 2).sum())
    # core/tests/test_core_plssvd.cpp:88-90
    assert abs(error - 10.5762741916562) < 2e-7
    assert abs(m["sigma"][0] - 119.561004785789) < 2e-7
    assert m["W"][0].shape == (1, 2) and m["W"][1].shape == (2, 2)


def test_simpls_known_answers():
    # core/tests/test_core_simpls.cpp:17-37
    vals = np.array([-3, -2, -1, 0, 0, 1, 2, 3, 1, -1, 1, -1, 1, -1, 1, -1,
                     -1, 2, -2, 1, 1, -2, 2, -1], dtype=np.float64)
    x = vals.reshape(3, 8).T
    coef = np.zeros((3, 3))
    coef[0, 0], coef[1, 0] = 1.5, -0.5
    coef[0, 1], coef[1, 1] = -0.75, 2.0
    coef[0, 2], coef[1, 2] = 0.25, 1.25
    y = x @ coef
    m = O.simpls_fit(x, y, ncomp=2, scaling=3, reorthogonalize=True)
    pred = O.simpls_predict(m, x, 2)
    rel = np.sqrt(((pred - y) ** 2).sum() / (y ** 2).sum())
    assert rel < 1e-8  # :84-88
    assert np.allclose(m["T"].T @ m["T"], np.eye(2), atol=1e-8)  # :102-117
    assert np.allclose(m["V"].T @ m["V"], np.eye(2), atol=1e-8)


def test_lda_known_answers():
    # core/tests/test_core_lda.cpp:8-31 (double instead of float)
    labels = np.array([1, 1, 1, 1, 2, 2, 2, 2])
    s = np.zeros((8, 3))
    for r in range(8):
        s[r, 0] = (-2.0 if r < 4 else 2.0) + 0.1 * (r % 4)
        s[r, 1] = 0.2 * r
        s[r, 2] = s[r, 1]
    models = O.lda_train(s, labels, 2, [1, 3])
    assert models[0]["linear"].shape == (2, 1)
    assert models[1]["linear"].shape == (2, 3)
    assert models[1]["ridge"] > 0
    pred = O.row_argmax(O.lda_discriminants(models[1], s))
    assert np.array_equal(pred, labels)


def test_topk_tie_rule():
    v = np.array([[1.0, 3.0, 3.0, 0.0], [2.0, 2.0, 2.0, 2.0]])
    assert O.topk(v, 2).tolist() == [[2, 3], [1, 2]]
    assert O.row_argmax(v).tolist() == [2, 1]


def test_permutation_pvalue():
    # R/main.R:2702-2718: (b + 1) / (B + 1) over finite values
    assert O.permutation_pvalue([0.1, 0.5, np.nan, 0.9], 0.5) == (2 + 1) / (3 + 1)
    assert O.permutation_pvalue([0.1, 0.5, 0.9], 0.5, lower_tail=True) == 3 / 4
    assert np.isnan(O.permutation_pvalue([np.nan], 0.5))


def label_fixture():
    # core/tests/test_core_classification.cpp:13-19: x(row, col) = 1 + row + 10 col
    # (4 x 3), classes 0, 1, 0, 1 (one-based here: 1, 2, 1, 2)
    x = np.array([[1 + r + 10 * c for c in range(3)] for r in range(4)], dtype=np.float64)
    return x, np.array([1, 2, 1, 2])


def test_label_crossprod_known_answers():
    x, lab = label_fixture()
    # centred label cross-product without scaling (:20-31): class sums minus
    # half the column total
    _, s, _, _, _, _ = O._prepare(x, None, lab, 2, 3)
    for c in range(3):
        zero, one = x[0, c] + x[2, c], x[1, c] + x[3, c]
        assert abs(s[c, 0] - (zero - 0.5 * (zero + one))) < 1e-12
        assert abs(s[c, 1] - (one - 0.5 * (zero + one))) < 1e-12
    # autoscaled (:33-44)
    _, s, centre, scale, ymean, _ = O._prepare(x, None, lab, 2, 2)
    assert abs(centre[0] - 2.5) < 1e-12
    assert abs(scale[0] - 1.2909944) < 1e-6
    assert abs(ymean[0] - 0.5) < 1e-12
    assert abs(s[0, 0] + 0.7745967) < 1e-6 and abs(s[0, 1] - 0.7745967) < 1e-6
