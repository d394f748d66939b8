"""int8 split product on the tensor cores vs its exact CPU emulation.

The digit products are exact integers on both sides and the FP64 epilogue
runs in the same order, so the device result must equal the emulation bit
for bit; its distance to the FP64 product stays inside the split's bound.
"""
import numpy as np
import pytest

from fastpls_b200 import api, workloads as W
from oracle import int8_split as Z

pytestmark = pytest.mark.gpu


def _operands(k, m, n, seed):
    g = W.rng(seed, 40)
    a = g.standard_normal((k, m)) * np.exp(g.standard_normal(m))[None, :]
    b = g.standard_normal((k, n)) * np.exp(g.standard_normal(n))[None, :]
    return a, b


# (tile width, CTA pair): single-CTA 128-row tiles of width 128/192/256 and
# CTA-pair 256-row tiles (tcgen05 cta_group::2) of width 192/256
TILES = [(128, 0), (192, 0), (256, 0), (192, 1), (256, 1)]


@pytest.mark.parametrize("tile_n,pair", TILES)
@pytest.mark.parametrize("digits", [1, 2, 3, 4, 5, 6, 7])
def test_bit_exact_against_emulation(digits, tile_n, pair):
    a, b = _operands(300, 200, 77 + tile_n, 1 + digits)
    got = api.int8_crossprod(a, b, digits=digits, tile_n=tile_n, pair=pair)
    ref = Z.product(a.T, b.T, digits, Z.pass_diagonals(tile_n))
    assert np.array_equal(got, ref)
    assert np.all(np.abs(got - a.T @ b) <= Z.error_bound(a.T, b.T, digits))


@pytest.mark.parametrize("tile_n,pair", TILES)
@pytest.mark.parametrize("k,m,n", [(1, 1, 1), (64, 128, 128), (65, 129, 257),
                                   (1000, 3, 300), (0, 5, 6), (96, 200, 450),
                                   (160, 513, 97)])
def test_shapes(k, m, n, tile_n, pair):
    a, b = _operands(k, m, n, 7)
    got = api.int8_crossprod(a, b, digits=6, tile_n=tile_n, pair=pair)
    assert np.array_equal(got, Z.product(a.T, b.T, 6, Z.pass_diagonals(tile_n)))


def test_width_choice_stays_accurate():
    # tile shape chosen for the shape (2010 columns); accuracy bound only
    a, b = _operands(600, 500, 2010, 17)
    got = api.int8_crossprod(a, b, digits=6)
    assert np.all(np.abs(got - a.T @ b) <= Z.error_bound(a.T, b.T, 6))


def test_pair_rejects_symmetric_and_narrow_tiles():
    a, _ = _operands(64, 40, 1, 19)
    with pytest.raises(RuntimeError):
        api.int8_crossprod(a, None, digits=6, pair=1)
    with pytest.raises(RuntimeError):
        api.int8_crossprod(a, a, digits=6, tile_n=128, pair=1)


def test_symmetric_lower_tiles_mirrored():
    a, _ = _operands(500, 300, 1, 9)
    got = api.int8_crossprod(a, None, digits=6)
    ref = Z.product(a.T, a.T, 6)
    assert np.array_equal(got, ref)
    assert np.array_equal(got, got.T)


def test_k_segments_keep_int32_exact():
    # digits 7: segments of 19008 k; 20000 needs two launches accumulating C
    a, b = _operands(20000, 40, 24, 11)
    for tile_n, pair in ((128, 0), (192, 0), (256, 1)):
        got = api.int8_crossprod(a, b, digits=7, tile_n=tile_n, pair=pair)
        assert np.array_equal(got, Z.product(a.T, b.T, 7, Z.pass_diagonals(tile_n)))


def test_zero_and_tiny_rows():
    a, b = _operands(200, 130, 20, 13)
    a[:, 5] = 0.0
    a[:, 6] = 1e-300
    b[:, 3] = 0.0
    for tile_n, pair in ((128, 0), (192, 1)):
        got = api.int8_crossprod(a, b, digits=6, tile_n=tile_n, pair=pair)
        assert np.array_equal(got, Z.product(a.T, b.T, 6, Z.pass_diagonals(tile_n)))
    assert np.all(got[5] == 0.0) and np.all(got[:, 3] == 0.0)


def test_non_finite_input_is_an_error():
    a, b = _operands(100, 10, 10, 15)
    a[3, 4] = np.nan
    with pytest.raises(RuntimeError, match="non-finite"):
        api.int8_crossprod(a, b, digits=6)
