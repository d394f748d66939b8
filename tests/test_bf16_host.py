"""BF16 bit conversion used for precision-16 predictors (host side)."""
import numpy as np
import torch

from fastpls_b200 import api


def test_to_bf16_matches_round_to_nearest_even():
    r = np.random.default_rng(5)
    x = np.concatenate([
        r.standard_normal(50000).astype(np.float32) * np.float32(1e3),
        np.exp(r.uniform(-80, 80, 20000)).astype(np.float32),
        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, np.inf, -np.inf, 1e-40], np.float32),
    ])
    want = torch.from_numpy(x).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(api.to_bf16(x), want)
    back = api.from_bf16(want)
    assert np.array_equal(back, torch.from_numpy(want.view(np.int16)).view(torch.bfloat16).float().numpy())


def test_nan_stays_nan_and_bits_pass_through():
    b = api.to_bf16(np.array([np.nan, -np.nan], np.float32))
    assert np.isnan(api.from_bf16(b)).all()
    bits = np.array([0x3F80, 0xC000], np.uint16)
    assert api.to_bf16(bits) is bits
    assert np.array_equal(api.from_bf16(bits), np.array([1.0, -2.0], np.float32))


def test_xmat_is_column_major_bits():
    x = np.arange(12, dtype=np.float32).reshape(3, 4)
    m = api._xmat(x, 16)
    assert m.dtype == np.uint16 and m.flags.f_contiguous and m.shape == (3, 4)
    assert np.array_equal(api.from_bf16(m).reshape(3, 4), x)
