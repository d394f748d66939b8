"""The no-allocation cross-product entry point (fastpls_b200_crossprod_noalloc).

It serves callers that cannot let the library allocate device memory (their
host owns every byte of GPU memory through its own pool or budget, or they
must not stall on the allocator): they hand over device buffers and the
library's partial sums live in a fixed file-scope device array. The test
checks its output against the existing fastpls_cuda_gemm entry point on two
consecutive calls (the second with new right-hand sides, so stale scratch
contents would show), against a host FP64 product on a shape whose partial
sums only fit as fewer, taller row chunks, and that oversized requests are
refused cleanly.
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, xd, precision, n, p, vd, nb, outd):
    err = C.create_string_buffer(256)
    rc = lib.fastpls_b200_crossprod_noalloc(
        C.c_void_p(xd.data_ptr()), precision, n, p, n, C.c_void_p(vd.data_ptr()),
        n, nb, C.c_void_p(outd.data_ptr()), p, None, err, C.c_size_t(256))
    return rc, err.value.decode()


def _reference(lib, x64, v):
    # existing entry point: fastpls_cuda_gemm(left = X^T, right = V), FP64
    left = np.asfortranarray(x64.T)
    right = np.asfortranarray(v)
    out = np.zeros((left.shape[0], right.shape[1]), order="F")
    err = C.create_string_buffer(256)
    rc = lib.fastpls_cuda_gemm(left.ctypes.data_as(C.c_void_p),
                               right.ctypes.data_as(C.c_void_p), 64,
                               left.shape[0], left.shape[1], right.shape[1],
                               out.ctypes.data_as(C.c_void_p), err, C.c_size_t(256))
    assert rc == 0, err.value
    return out


@pytest.mark.parametrize("precision", [64, 32])
def test_noalloc_crossprod_matches_gemm_entry_point(precision):
    import torch

    from fastpls_b200 import _lib
    lib = _lib.load()
    n, p, nb = 3001, 517, 5
    rng = np.random.default_rng(7)
    dt = np.float64 if precision == 64 else np.float32
    x = np.asfortranarray(rng.standard_normal((n, p)).astype(dt))
    x64 = x.astype(np.float64)
    dev = torch.device("cuda", 0)
    # column-major n x p on the device: a (p, n) row-major tensor
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).to(dev)
    outd = torch.zeros((nb, p), dtype=torch.float64, device=dev)
    for call in range(2):
        v = np.asfortranarray(rng.standard_normal((n, nb)))
        vd = torch.from_numpy(np.ascontiguousarray(v.T)).to(dev)
        rc, msg = _noalloc(lib, xd, precision, n, p, vd, nb, outd)
        assert rc == 0, msg
        got = outd.cpu().numpy().T
        want = _reference(lib, x64, v)
        rel = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert rel < 1e-12, (call, rel)


def test_noalloc_tall_chunks_match_host_product():
    """p * nb = 524288 doubles leaves room for 4 row chunks: 5000 rows run as
    4 chunks of 1250 rows, each staged through shared memory 192 rows at a
    time, so every slot is written once and then accumulated into."""
    import torch

    from fastpls_b200 import _lib
    lib = _lib.load()
    n, p, nb = 5000, 16384, 32
    rng = np.random.default_rng(11)
    x = rng.standard_normal((n, p), dtype=np.float32)
    dev = torch.device("cuda", 0)
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).to(dev)
    outd = torch.zeros((nb, p), dtype=torch.float64, device=dev)
    x64 = x.astype(np.float64)
    for call in range(2):
        v = rng.standard_normal((n, nb))
        vd = torch.from_numpy(np.ascontiguousarray(v.T)).to(dev)
        rc, msg = _noalloc(lib, xd, 32, n, p, vd, nb, outd)
        assert rc == 0, msg
        got = outd.cpu().numpy().T
        want = x64.T @ v
        rel = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert rel < 1e-12, (call, rel)


def test_noalloc_rejects_requests_beyond_its_scratch():
    import torch

    from fastpls_b200 import _lib
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    n, p, nb = 4, 2097152 // 4 + 1, 4   # p * nb just above 2097152 doubles
    xd = torch.zeros(1, dtype=torch.float64, device=dev)
    vd = torch.zeros(n * nb, dtype=torch.float64, device=dev)
    outd = torch.zeros(1, dtype=torch.float64, device=dev)
    rc, msg = _noalloc(lib, xd, 64, n, p, vd, nb, outd)
    assert rc == 1 and "scratch capacity" in msg
