"""Host-to-device uploads of caller buffers: a pageable, misaligned source
above the staging threshold (several pinned chunks and a ragged last one)
gives the same model, bit for bit, as the same values in pinned memory
(one direct copy), and both agree with the oracle."""
import numpy as np
import pytest
import torch

from fastpls_b200 import api, workloads as W
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu


def test_staged_upload_matches_pinned_source():
    n, p, q, a = 3001, 9001, 3, 6      # 108 MB of FP32: 6 full 16 MB chunks and a ragged one
    x, y = W.latent_regression(n, p, q, 4, 0.4, 41, dtype=np.float32)
    # pageable, 4 bytes past a 16-byte boundary
    buf = np.empty(n * p + 1, dtype=np.float32)
    xv = buf[1:].reshape((n, p), order="F")
    xv[...] = x
    assert xv.ctypes.data % 16 == 4 and xv.flags.f_contiguous
    # pinned
    pin = torch.empty(n * p, dtype=torch.float32).pin_memory()
    xp = pin.numpy().reshape((n, p), order="F")
    xp[...] = x
    probe = np.asfortranarray(x[::7])
    m1 = api.fit_resident(xv, y, ncomp=a, precision=32)
    m2 = api.fit_resident(xp, y, ncomp=a, precision=32)
    for f in (0, 1, 2):
        assert np.array_equal(m1.export(f), m2.export(f)), f
    got = m1.predict_path(probe, [1, a])
    assert np.array_equal(got, m2.predict_path(probe, [1, a]))
    m1.close()
    m2.close()
    ref = O.simpls_fit(x.astype(np.float64), y.astype(np.float64), ncomp=a)
    want = O.simpls_predict(ref, probe.astype(np.float64), a)
    assert O.rel_err(got[1].astype(np.float64), want) < 1e-5


def test_concurrent_staged_uploads_in_the_server():
    """Fits above the staging threshold submitted to four server workers at
    once (their uploads share the pooled pinned slots and copy threads) give
    the models of the same fits made alone, bit for bit."""
    specs = [(2100 + 97 * i, 1500 + 53 * i, 1 + i % 3, 4 + i % 3) for i in range(6)]  # 12-20 MB each
    data = [W.latent_regression(n, p, q, 4, 0.4, 900 + i, dtype=np.float32)
            for i, (n, p, q, a) in enumerate(specs)]
    srv = api.Server(workers=4)
    tickets = [srv.submit_fit(x, y, ncomp=a, precision=32)
               for (x, y), (n, p, q, a) in zip(data, specs)]
    for t in tickets:
        srv.wait(t)
    for i, ((x, y), (n, p, q, a)) in enumerate(zip(data, specs)):
        probe = np.asfortranarray(x[::11])
        got, _, _ = srv.wait(srv.submit_predict(tickets[i], probe, [a]))
        alone = api.fit_resident(x, y, ncomp=a, precision=32)
        assert np.array_equal(got, alone.predict_path(probe, [a])), i
        alone.close()
        srv.release(tickets[i])
    srv.close()
