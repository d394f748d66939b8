import numpy as np

from fastpls_b200 import workloads as W


def test_generator_is_deterministic():
    a = W.latent_regression(30, 20, 2, 3, 0.5, 4)
    b = W.latent_regression(30, 20, 2, 3, 0.5, 4)
    assert all(np.array_equal(u, v) for u, v in zip(a, b))
    x, _ = a
    assert x.flags.f_contiguous and np.allclose(x.mean(axis=0), 0, atol=1e-5)


def test_uneven_folds_cv_configuration():
    folds = W.uneven_folds(5000, 10, 3)
    sizes = np.bincount(folds)[1:]
    assert sizes.sum() == 5000 and len(sizes) == 10
    assert sizes.min() >= 480 and sizes.max() <= 520
    assert len(set(sizes.tolist())) > 1  # uneven


def test_permutations_are_permutations():
    p = W.permutations(100, 5, 1)
    assert p.shape == (5, 100)
    for row in p:
        assert np.array_equal(np.sort(row), np.arange(100))
    assert W.permutations(10, 0, 1).shape == (0, 10)


def test_classification_labels_one_based():
    _, lab = W.latent_classification(200, 10, 5, 3, 0.1, 2)
    assert lab.min() >= 1 and lab.max() <= 5
