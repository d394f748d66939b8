"""Cross-validation entry points and the batched permutation engine vs the oracle."""
import numpy as np
import pytest

from fastpls_b200 import api, workloads as W
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method,family", [("simpls", 3), ("plssvd", 1)])
@pytest.mark.parametrize("scaling", [1, 2])
def test_cv_regression(method, family, scaling):
    x, y = W.latent_regression(240, 150, 3, 4, 0.4, 21, dtype=np.float64)
    folds = W.uneven_folds(240, 5, 21)
    pre = [1, 2, 3] if method == "plssvd" else [1, 2, 4, 6, 8]
    got = api.cv_regression(x, y, folds, pre, scaling=scaling, method=method,
                            store_predictions=True)
    ref = O.cv_regression(x, y, folds, pre, scaling=scaling, family=family,
                          store_predictions=True)
    for key in ("q2", "rmsd", "observed_r2"):
        assert np.allclose(got[key], ref[key], rtol=1e-9, atol=1e-11), key
    assert O.rel_err(got["predictions"], ref["predictions"]) < 1e-9
    assert list(got["status"]) == [1] * 5


@pytest.mark.parametrize("lda", [False, True])
def test_cv_classification(lda):
    x, lab = W.latent_classification(260, 120, 4, 3, 0.5, 23, dtype=np.float64)
    folds = W.uneven_folds(260, 4, 23)
    pre = [1, 2, 3]
    got = api.cv_classification(x, lab, 4, folds, pre, lda=lda,
                                store_predictions=True)
    ref = O.cv_classification(x, lab, 4, folds, pre, head=int(lda),
                              store_predictions=True)
    assert np.array_equal(got["predictions"], ref["predictions"])
    assert np.allclose(got["metrics"], ref["metrics"])


# digits 0: products with the shared Gram as FP64 DMMA GEMMs (FP64 parity);
# digits 6: int8 split products on the tensor cores, held to the 1e-5
# relative tolerance of the mixed-precision path.
@pytest.mark.parametrize("digits,rtol", [(0, 1e-9), (6, 1e-5)])
@pytest.mark.parametrize("scaling", [1, 2, 3])
def test_batched_cv_permutation(scaling, digits, rtol):
    n, p = 300, 420
    x, y = W.latent_regression(n, p, 3, 5, 0.3, 31, dtype=np.float32)
    folds = W.uneven_folds(n, 5, 31)
    perms = W.permutations(n, 3, 31)
    pre = [1, 2, 3, 5, 8]
    got = api.cv_permutation(x, y, folds, perms, pre, scaling=scaling, precision=32,
                             digits=digits)
    x64, y64 = x.astype(np.float64), y.astype(np.float64)
    for b in range(4):
        yb = y64 if b == 0 else y64[perms[b - 1]]
        ref = O.cv_regression(x64, yb, folds, pre, scaling=scaling, family=3)
        for key in ("q2", "rmsd", "observed_r2"):
            assert np.allclose(got[key][b], ref[key], rtol=rtol, atol=rtol * 1e-2), (b, key)


def test_batched_matches_plain_cv():
    n, p = 200, 90
    x, y = W.latent_regression(n, p, 2, 3, 0.3, 41, dtype=np.float64)
    folds = W.uneven_folds(n, 4, 41)
    pre = [1, 2, 3, 4]
    plain = api.cv_regression(x, y, folds, pre)
    batched = api.cv_permutation(x, y, folds, None, pre, precision=64, digits=0)
    assert np.allclose(batched["q2"][0], plain["q2"], rtol=1e-10, atol=1e-12)


# the register-resident score kernel holds ceil(n / 256) rows per thread in
# 8/16/20/24/32-row variants; larger n uses the general kernel
@pytest.mark.parametrize("n", [1500, 4600, 7000, 9000])
def test_batched_row_variants(n):
    p = 120
    x, y = W.latent_regression(n, p, 2, 4, 0.3, 43, dtype=np.float64)
    folds = W.uneven_folds(n, 4, 43)
    perms = W.permutations(n, 1, 43)
    pre = [1, 2, 4, 7]
    got = api.cv_permutation(x, y, folds, perms, pre, precision=64, digits=0)
    for b in range(2):
        yb = y if b == 0 else y[perms[b - 1]]
        ref = O.cv_regression(x, yb, folds, pre, family=3)
        for key in ("q2", "rmsd", "observed_r2"):
            assert np.allclose(got[key][b], ref[key], rtol=1e-9, atol=1e-11), (b, key)


@pytest.mark.parametrize("lanes", [1, 2, 3])
@pytest.mark.parametrize("digits,rtol", [(0, 1e-9), (6, 1e-5)])
def test_batched_lanes(digits, rtol, lanes):
    # 5 folds x (1 + 19) response orders = 100 instances: up to three stream
    # lanes of >= 32 instances; results must not depend on the lane count
    old = api.batch_lanes()
    api.set_batch_lanes(lanes)
    n, p = 260, 150
    x, y = W.latent_regression(n, p, 2, 4, 0.3, 47, dtype=np.float64)
    folds = W.uneven_folds(n, 5, 47)
    perms = W.permutations(n, 19, 47)
    pre = [1, 3, 6]
    try:
        got = api.cv_permutation(x, y, folds, perms, pre, precision=64, digits=digits)
    finally:
        api.set_batch_lanes(old)
    for b in (0, 7, 19):
        yb = y if b == 0 else y[perms[b - 1]]
        ref = O.cv_regression(x, yb, folds, pre, family=3)
        for key in ("q2", "rmsd", "observed_r2"):
            assert np.allclose(got[key][b], ref[key], rtol=rtol, atol=rtol * 1e-2), (b, key)


@pytest.mark.parametrize("q", [1, 5])
def test_batched_response_counts(q):
    # the deflation keeps its Kw^T C sums in registers for q <= 4 and has a
    # general form for larger q
    n, p = 220, 130
    x, y = W.latent_regression(n, p, q, 4, 0.3, 53, dtype=np.float64)
    folds = W.uneven_folds(n, 4, 53)
    perms = W.permutations(n, 2, 53)
    pre = [1, 2, 5]
    got = api.cv_permutation(x, y, folds, perms, pre, precision=64, digits=0)
    for b in range(3):
        yb = y if b == 0 else y[perms[b - 1]]
        ref = O.cv_regression(x, yb, folds, pre, family=3)
        for key in ("q2", "rmsd", "observed_r2"):
            assert np.allclose(got[key][b], ref[key], rtol=1e-9, atol=1e-11), (b, key)


@pytest.mark.parametrize("digits", [0, 6])
@pytest.mark.parametrize("scaling", [1, 2])
def test_batched_classification_permutations(digits, scaling):
    n, p, classes = 260, 150, 4
    x, lab = W.latent_classification(n, p, classes, 3, 0.5, 41, dtype=np.float32)
    lab = lab.copy()
    lab[7] = 5          # a fifth class with one row: absent from four training folds
    classes = 5
    folds = W.uneven_folds(n, 5, 41)
    perms = W.permutations(n, 3, 41)
    pre = [1, 2, 4, 6]
    got = api.cv_permutation_classification(x, lab, classes, folds, perms, pre,
                                            scaling=scaling, digits=digits)
    x64 = x.astype(np.float64)
    for b in range(4):
        lb = lab if b == 0 else lab[perms[b - 1]]
        want = O.cv_classification(x64, lb, classes, folds, pre, scaling=scaling)["metrics"]
        # labels are bit-exact with int8 products too: the argmax guard
        # refits instances with near-tied held-out scores in FP64
        assert np.array_equal(got["accuracy"][b], want), (b, got["accuracy"][b], want)
    assert list(got["status"]) == [1] * 5


@pytest.mark.parametrize("scaling", [1, 2])
def test_argmax_guard_refits_every_marked_instance(scaling):
    """A margin of 1e30 marks every instance with two or more active classes, so
    the whole run is refitted with FP64 products: the accuracies must then be
    identical to the FP64-product run, and the refit count must be every
    instance."""
    n, p, classes = 240, 120, 3
    x, lab = W.latent_classification(n, p, classes, 3, 0.5, 43, dtype=np.float64)
    folds = W.uneven_folds(n, 4, 43)
    perms = W.permutations(n, 5, 43)
    pre = [1, 2, 5]
    fp64 = api.cv_permutation_classification(x, lab, classes, folds, perms, pre,
                                             scaling=scaling, digits=0)
    assert api.guard_refits() == 0
    old = api.argmax_guard()
    api.set_argmax_guard(1e30)
    try:
        got = api.cv_permutation_classification(x, lab, classes, folds, perms, pre,
                                                scaling=scaling, digits=6)
        refits = api.guard_refits()
    finally:
        api.set_argmax_guard(old)
    assert refits == 6 * 4
    assert np.array_equal(got["accuracy"], fp64["accuracy"])


def test_batched_classification_ten_classes_bit_exact():
    """The PLS-SVD + LDA configuration's label shape (10 classes from the
    argmax of latent scores) at a reduced size, 6-digit products: held-out
    accuracies equal the FP64 oracle's for every permutation and prefix."""
    n, p, classes = 600, 400, 10
    x, lab = W.latent_classification(n, p, classes, 20, 0.1, 2, dtype=np.float32)
    folds = W.uneven_folds(n, 5, 2)
    perms = W.permutations(n, 4, 2)
    pre = [1, 3, 6, 9]
    got = api.cv_permutation_classification(x, lab, classes, folds, perms, pre, digits=6)
    x64 = x.astype(np.float64)
    for b in range(5):
        lb = lab if b == 0 else lab[perms[b - 1]]
        want = O.cv_classification(x64, lb, classes, folds, pre)["metrics"]
        assert np.array_equal(got["accuracy"][b], want), (b, got["accuracy"][b], want)


@pytest.mark.parametrize("lda", [False, True])
def test_batched_classification_single_class_folds(lda):
    """A training fold with one class predicts that class for its held-out
    rows (the reference's status-4 fold); the other folds are fitted."""
    n = 120
    x, _ = W.latent_classification(n, 40, 2, 3, 0.5, 42, dtype=np.float32)
    folds = W.uneven_folds(n, 4, 42)
    lab = np.ones(n, dtype=np.int32)
    lab[folds == 1] = 2          # class 2 only in fold 1: its training rows hold one class
    lab[:5] = 2
    perms = W.permutations(n, 2, 42)
    pre = [1, 2]
    got = api.cv_permutation_classification(x, lab, 2, folds, perms, pre, digits=0, lda=lda)
    x64 = x.astype(np.float64)
    for b in range(3):
        lb = lab if b == 0 else lab[perms[b - 1]]
        want = O.cv_classification(x64, lb, 2, folds, pre, head=1 if lda else 0)
        assert np.array_equal(got["accuracy"][b], want["metrics"]), b
        if b == 0:
            assert list(got["status"]) == list(want["status"])


def test_batched_graph_replay_and_schedules_bit_identical():
    """The second call of a shape replays the group's captured CUDA graph
    (no new capture); the tuned schedule, every fixed lane count and the
    FP64-free default give bit-identical results, since the candidate tile
    widths (192, 256) combine the digit diagonals in one FP64 order and
    lanes only partition the instances."""
    n, p = 300, 160
    x, y = W.latent_regression(n, p, 3, 4, 0.3, 61, dtype=np.float32)
    folds = W.uneven_folds(n, 5, 61)
    perms = W.permutations(n, 99, 61)      # 500 instances: up to 4 lanes of 125
    pre = [1, 2, 4, 7]
    api.release_workspace()
    first = api.cv_permutation(x, y, folds, perms, pre, precision=32, digits=6)
    s1 = api.batched_stats()
    assert s1["groups"] == 1 and s1["graph_captures"] >= 1
    second = api.cv_permutation(x, y, folds, perms, pre, precision=32, digits=6)
    s2 = api.batched_stats()
    assert s2["graph_replays"] == 1 and s2["graph_captures"] == 0 and s2["tuned"] == 0
    for key in ("q2", "rmsd", "observed_r2"):
        assert np.array_equal(first[key], second[key]), key
    old_tune, old_lanes = api.autotune(), api.batch_lanes()
    try:
        api.set_autotune(False)
        for lanes in (1, 2, 3, 4):
            api.set_batch_lanes(lanes)
            got = api.cv_permutation(x, y, folds, perms, pre, precision=32, digits=6)
            assert api.batched_stats()["lanes"] == lanes
            for key in ("q2", "rmsd", "observed_r2"):
                assert np.array_equal(first[key], got[key]), (lanes, key)
    finally:
        api.set_autotune(old_tune)
        api.set_batch_lanes(old_lanes)
    # new inputs of the same shape replay the same graph and match the oracle
    x2, y2 = W.latent_regression(n, p, 3, 4, 0.3, 62, dtype=np.float32)
    got = api.cv_permutation(x2, y2, folds, perms, pre, precision=32, digits=6)
    assert api.batched_stats()["graph_captures"] == 0
    for b in (0, 50, 99):
        yb = y2 if b == 0 else y2[perms[b - 1]]
        ref = O.cv_regression(x2.astype(np.float64), yb.astype(np.float64), folds, pre)
        assert np.allclose(got["q2"][b], ref["q2"], rtol=1e-5, atol=1e-7), b


@pytest.mark.parametrize("digits", [0, 6])
@pytest.mark.parametrize("scaling", [1, 2])
def test_batched_classification_lda_head(digits, scaling):
    """LDA on the latent scores per (fold, permutation) instance, as the
    reference's classification CV with the LDA head (compacted active
    classes per training fold): accuracies equal the FP64 oracle's for every
    permutation and prefix, including a class absent from most training
    folds."""
    n, p, classes = 300, 160, 4
    x, lab = W.latent_classification(n, p, classes, 4, 0.5, 44, dtype=np.float32)
    lab = lab.copy()
    lab[11] = 5
    classes = 5
    folds = W.uneven_folds(n, 5, 44)
    perms = W.permutations(n, 3, 44)
    pre = [1, 2, 4, 7]
    got = api.cv_permutation_classification(x, lab, classes, folds, perms, pre,
                                            scaling=scaling, digits=digits, lda=True)
    x64 = x.astype(np.float64)
    for b in range(4):
        lb = lab if b == 0 else lab[perms[b - 1]]
        want = O.cv_classification(x64, lb, classes, folds, pre, scaling=scaling, head=1)["metrics"]
        assert np.array_equal(got["accuracy"][b], want), (b, got["accuracy"][b], want)
    # the argmax head on the same inputs is a different classifier
    arg = api.cv_permutation_classification(x, lab, classes, folds, perms, pre,
                                            scaling=scaling, digits=digits)
    assert arg["accuracy"].shape == got["accuracy"].shape


@pytest.mark.parametrize("digits", [0, 6])
def test_batched_classification_candidate_blocks(digits):
    """Training folds with n_train p classes >= 5e8 and 4+ components take
    candidate blocks (min(64, components, p, classes) directions from one
    decomposition, src/cuda_resident_simpls.cuh:144-153): 2400 x 8000 training
    rows with 28 active classes and 10 components take all ten directions
    from the first decomposition. Accuracies equal the FP64 oracle run with
    the same block rule, for the observed and permuted labels."""
    n, p, classes = 3000, 8000, 30
    x, lab = W.latent_classification(n, p, classes, 12, 0.5, 45, dtype=np.float32)
    folds = W.uneven_folds(n, 5, 45)
    perms = W.permutations(n, 2, 45)
    pre = [1, 3, 8, 10]
    ntr = n - int(np.sum(folds == 1))
    active = np.unique(lab[folds != 1]).size
    assert ntr * p * active >= 5e8
    assert O.simpls_block_size(ntr, p, active, 10, True) == 10
    got = api.cv_permutation_classification(x, lab, classes, folds, perms, pre, digits=digits)
    x64 = x.astype(np.float64)
    for b in range(3):
        lb = lab if b == 0 else lab[perms[b - 1]]
        want = O.cv_classification(x64, lb, classes, folds, pre)["metrics"]
        assert np.array_equal(got["accuracy"][b], want), (b, got["accuracy"][b], want)
