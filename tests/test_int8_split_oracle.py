"""The int8 split emulation (oracle/int8_split.py) on the CPU: digit
reconstruction, the error bound against the FP64 product, and the int32
headroom rule of its k segments."""
import numpy as np
import pytest

from fastpls_b200 import workloads as W
from oracle import int8_split as Z


def _rows(r, k, seed):
    g = W.rng(seed, 41)
    return g.standard_normal((r, k)) * np.exp(2.0 * g.standard_normal(r))[:, None]


@pytest.mark.parametrize("digits", [1, 3, 6, 7])
def test_digits_reconstruct_rows(digits):
    x = _rows(50, 300, digits)
    planes, scale = Z.split(x, digits)
    for d in planes:
        assert np.all(np.abs(d) <= 127) and np.all(d == np.rint(d))
    back = sum(d * 254.0 ** -s for s, d in enumerate(planes)) / 127.0 * scale[:, None]
    tail = 0.5 / (127.0 * 254.0 ** (digits - 1)) * scale[:, None]
    assert np.all(np.abs(back - x) <= tail * (1 + 1e-9) + 1e-15 * np.abs(x))


@pytest.mark.parametrize("digits", [1, 2, 4, 6, 7])
def test_product_within_bound(digits):
    a, b = _rows(40, 500, 5), _rows(30, 500, 6)
    got = Z.product(a, b, digits)
    assert np.all(np.abs(got - a @ b.T) <= Z.error_bound(a, b, digits))


def test_six_digits_near_fp64():
    a, b = _rows(20, 2000, 7), _rows(20, 2000, 8)
    ref = a @ b.T
    scale = np.outer(np.abs(a).max(1), np.abs(b).max(1)) * 2000
    assert np.max(np.abs(Z.product(a, b, 6) - ref) / scale) < 2.0 ** -46


def test_segments_cover_k_and_sum_exactly():
    # worst case digits: every product at 127^2; a segment must stay < 2^31
    for digits in range(1, 8):
        seg = max(1, (2147483647 // (16129 * digits)) // Z.KB) * Z.KB
        assert digits * seg * 16129 < 2 ** 31
    a, b = _rows(3, 20000, 9), _rows(2, 20000, 10)
    assert np.all(np.abs(Z.product(a, b, 7) - a @ b.T) <= Z.error_bound(a, b, 7))
