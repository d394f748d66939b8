"""Bounded waits: a wait that nothing completes runs out, the kernel reports
it through its error flag and returns, and the device stays usable.

No GPU fault is involved: the int8 product's producer withholds its last
pipeline stage (so the MMA issuer's wait for it runs out after a short
bound), and one CTA of the persistent fit leaves before its first barrier
(so the other CTAs' barrier waits run out). Both hooks only skip work; every
copy and MMA that is issued is waited for before a CTA exits."""
import ctypes as C

import numpy as np
import pytest

from fastpls_b200 import _lib, api, workloads as W
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu

SHORT = 20_000_000   # clocks: about 10 ms at B200 clocks


def test_int8_product_wait_runs_out_and_device_recovers():
    lib = _lib.load()
    rng = np.random.default_rng(5)
    a = rng.standard_normal((700, 300))
    b = rng.standard_normal((700, 260))
    lib.fastpls_b200_int8_wait_test(1, C.c_longlong(SHORT))
    try:
        with pytest.raises(_lib.FastplsError, match="timed out"):
            api.int8_crossprod(a, b, digits=6, tile_n=192, pair=0)
    finally:
        lib.fastpls_b200_int8_wait_test(0, C.c_longlong(0))
    got = api.int8_crossprod(a, b, digits=6, tile_n=192, pair=0)
    assert O.rel_err(got, a.T @ b) < 1e-13


def test_persistent_barrier_wait_runs_out_and_device_recovers():
    lib = _lib.load()
    x, y = W.latent_regression(2000, 3000, 3, 4, 0.4, 91, dtype=np.float64)
    lib.fastpls_b200_persistent_wait_test(1, C.c_longlong(SHORT))
    try:
        with pytest.raises(_lib.FastplsError):
            api.fit_resident(x, y, ncomp=4, precision=64)
    finally:
        lib.fastpls_b200_persistent_wait_test(0, C.c_longlong(0))
    m = api.fit_resident(x, y, ncomp=4, precision=64)
    ref = O.simpls_fit(x, y, ncomp=4)
    assert O.rel_err(m.export(0) @ m.export(1).T, ref["R"] @ ref["Q"].T) < 1e-9
    m.close()
