"""Candidate blocks of SIMPLS directions (src/cuda_resident_simpls.cuh:144-153,
inst/include/fastpls/core/simpls.hpp:43-62 and :547-595): large classification
fits take several directions from one decomposition of the cross-product. The
numpy oracle is checked against the compiled reference core at a size that
triggers the rule."""
import numpy as np
import pytest

from fastpls_b200 import workloads as W
from oracle import pls_oracle as O
from oracle import ref

# n p q = 5e8 exactly: the smallest work the rule accepts
BLOCK_SHAPE = (4000, 2500, 50)


def test_block_size_rule():
    bs = O.simpls_block_size
    assert bs(4000, 2500, 50, 8, True) == 8
    assert bs(4000, 2500, 50, 100, True) == 50           # capped by q
    assert bs(4000, 2500, 50, 3, True) == 1              # fewer than 4 components
    assert bs(3999, 2500, 50, 8, True) == 1              # n p q below 5e8
    assert bs(4000, 2500, 50, 8, False) == 1             # FP64 regression
    assert bs(20000, 40, 2100, 8, True) == 1             # more than 2048 classes
    assert bs(100000, 3000, 100, 200, True) == 64        # block maximum
    assert bs(10, 2_100_000, 64, 8, False, fp32=True) == 8   # FP32 cross-covariance > 512 MiB
    assert bs(10, 2_000_000, 64, 8, False, fp32=True) == 1


def test_block_route_in_oracle_is_not_per_component():
    # the block route gives different weights from the per-component route
    x, lab = W.latent_classification(600, 90, 12, 4, 0.5, 3, dtype=np.float64)
    a = O.simpls_fit(x, labels=lab, classes=12, ncomp=8, block=8)
    b = O.simpls_fit(x, labels=lab, classes=12, ncomp=8, block=1)
    assert O.rel_err(a["R"] @ a["Q"].T, b["R"] @ b["Q"].T) > 1e-4
    # the first direction of a block is the dominant one either way
    assert O.rel_err(O.align_signs(a["R"][:, :1], b["R"][:, :1]), b["R"][:, :1]) < 1e-12


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_block_route_matches_reference():
    n, p, q = BLOCK_SHAPE
    x, lab = W.latent_classification(n, p, q, 50, 0.5, 11, dtype=np.float64)
    assert O.simpls_block_size(n, p, q, 8, True) == 8
    a = O.simpls_fit(x, labels=lab, classes=q, ncomp=8, scaling=1)
    b = ref.simpls_fit(x, labels=lab, classes=q, ncomp=8, scaling=1)
    assert a["R"].shape[1] == b["R"].shape[1] == 8
    assert O.rel_err(a["R"] @ a["Q"].T, b["R"] @ b["Q"].T) < 1e-8
    assert O.rel_err(O.align_signs(a["T"], b["T"]), b["T"]) < 1e-8
    one = O.simpls_fit(x, labels=lab, classes=q, ncomp=8, scaling=1, block=1)
    assert O.rel_err(one["R"] @ one["Q"].T, b["R"] @ b["Q"].T) > 1e-6
