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


def _residual(x, u, d, v):
    """max_j max(||x v_j - d_j u_j||, ||x^T u_j - d_j v_j||) / d_1
    (triplet_residual, inst/include/fastpls/core/audited_rsvd.hpp:103-143)."""
    f = np.linalg.norm(x @ v - u * d, axis=0)
    r = np.linalg.norm(x.T @ u - v * d, axis=0)
    return float(np.max(np.maximum(f, r)) / max(abs(d[0]), np.finfo(float).eps))


def test_fastsvd_audit_certifies_first_attempt():
    x, _ = W.latent_regression(400, 260, 1, 6, 0.05, 62, dtype=np.float64)
    u, d, v, info = api.fastsvd(x, 4, oversample=10, power=2, seed=3, audit=True)
    assert info["certified"] and not info["deterministic_fallback"]
    assert info["attempts"] == 1
    assert info["effective_oversample"] == 10 and info["effective_power"] == 2
    assert info["triplet_residual"] <= 1e-2 and info["omitted_direction_ratio"] <= 1.01
    assert _residual(x, u, d, v) <= info["triplet_residual"] * (1 + 1e-9) + 1e-15
    S = np.linalg.svd(x, compute_uv=False)
    assert np.allclose(d, S[:4], rtol=1e-9)


def test_fastsvd_audit_retries_a_flat_spectrum():
    # no sketch oversampling and no power steps on a slowly decaying spectrum:
    # the first attempt fails the audit; the escalated attempts certify
    rng = np.random.default_rng(9)
    n, p, k = 300, 200, 5
    qa, _ = np.linalg.qr(rng.standard_normal((n, p)))
    qb, _ = np.linalg.qr(rng.standard_normal((p, p)))
    s = np.concatenate([[20.0, 16.0, 13.0, 11.0, 10.0], 9.0 * 0.995 ** np.arange(p - 5)])
    x = (qa * s) @ qb.T
    u, d, v, info = api.fastsvd(x, k, oversample=0, power=0, seed=1, audit=True)
    assert info["certified"] and info["attempts"] >= 2
    assert info["effective_oversample"] >= 32 and info["effective_power"] >= 3
    assert info["effective_seed"] != 1
    assert np.allclose(d, s[:k], rtol=1e-4)
    assert _residual(x, u, d, v) <= 1e-2


def test_fastsvd_small_matrix_is_exact():
    rng = np.random.default_rng(4)
    x = rng.standard_normal((40, 5))
    u, d, v, info = api.fastsvd(x, 3, oversample=0, power=0, seed=1, audit=True)
    assert info["certified"] and info["deterministic_fallback"]
    U, S, Vt = np.linalg.svd(x, full_matrices=False)
    assert np.allclose(d, S[:3], rtol=1e-12)
    assert O.rel_err(O.align_signs(u, U[:, :3]), U[:, :3]) < 1e-10


@pytest.mark.parametrize("precision,tol", [(64, 1e-8), (32, 2e-3)])
def test_fastsvd_known_answer(precision, tol):
    # core/tests/test_core_operator_rsvd.cpp:140-178: a 10 x 8 matrix with
    # diagonal 8, 7, ..., 1, rank 2, oversample 6, one power step, seed 27
    x = np.zeros((10, 8))
    for i in range(8):
        x[i, i] = 8 - i
    u, d, v = api.fastsvd(x, 2, oversample=6, power=1, seed=27, precision=precision)
    assert u.shape == (10, 2) and v.shape == (8, 2)
    assert abs(d[0] - 8) < tol and abs(d[1] - 7) < tol
    for j in range(2):
        assert np.linalg.norm(x @ v[:, j] - d[j] * u[:, j]) / d[j] < tol
