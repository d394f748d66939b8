"""Serving loop: mixed fit / predict requests with continuous admission give
the same results as standalone calls (and as the oracle)."""
import numpy as np
import pytest

from fastpls_b200 import api, workloads as W
from oracle import pls_oracle as O

pytestmark = pytest.mark.gpu

SPECS = [  # (method, n, p, q, ncomp, classification)
    ("simpls", 300, 400, 3, 5, False),
    ("plssvd", 250, 180, 4, 3, False),
    ("opls", 200, 150, 2, 3, False),
    ("kernelpls", 180, 90, 2, 4, False),
    ("simpls", 240, 120, 3, 4, True),
    ("simpls", 500, 800, 5, 8, False),
]


def _data(i, method, n, p, q, cls):
    if cls:
        x, lab = W.latent_classification(n, p, q, 3, 0.4, 100 + i, dtype=np.float32)
        return x, None, lab
    x, y = W.latent_regression(n, p, q, 4, 0.4, 100 + i, dtype=np.float32)
    return x, y, None


def _kw(method, p):
    return dict(kernel="rbf", gamma=1.0 / p) if method == "kernelpls" else {}


@pytest.mark.parametrize("budget,workers,borrow", [(150 * 10**9, 4, True), (300 * 10**6, 2, True),
                                                    (150 * 10**9, 4, False)])
def test_mixed_requests_match_standalone(budget, workers, borrow):
    """Borrowed inputs (read in place, the default) and copied inputs give the
    same bits as standalone calls."""
    srv = api.Server(budget_bytes=budget, workers=workers, borrow=borrow)
    fits, preds = {}, {}
    for i, (method, n, p, q, a, cls) in enumerate(SPECS):
        x, y, lab = _data(i, method, n, p, q, cls)
        t = srv.submit_fit(x, y, labels=lab, classes=q if cls else None, ncomp=a,
                           method=method, precision=32, **_kw(method, p))
        fits[i] = t
    for i, (method, n, p, q, a, cls) in enumerate(SPECS):
        srv.wait(fits[i])
        xt, _, _ = _data(50 + i, method, 37 + i, p, q, False)
        for part in range(3):  # several requests per model: merged batches
            preds[(i, part)] = srv.submit_predict(fits[i], xt[part::3], [1, a])
    for (i, part), t in preds.items():
        got, qms, sms = srv.wait(t)
        method, n, p, q, a, cls = SPECS[i]
        x, y, lab = _data(i, method, n, p, q, cls)
        xt, _, _ = _data(50 + i, method, 37 + i, p, q, False)
        alone = api.fit_resident(x, y, labels=lab, classes=q if cls else None, ncomp=a,
                                 method=method, precision=32, **_kw(method, p))
        want = alone.predict_path(xt[part::3], [1, a])
        alone.close()
        assert np.array_equal(got, want), (i, part)  # bitwise: deterministic kernels
        assert qms >= 0 and sms >= 0
    for t in fits.values():
        srv.release(t)
    assert srv.stats()["resident_models"] == 0
    srv.close()


def test_served_simpls_matches_oracle():
    srv = api.Server(workers=2)
    x, y = W.latent_regression(260, 300, 3, 4, 0.4, 7, dtype=np.float64)
    xt, _ = W.latent_regression(40, 300, 3, 4, 0.4, 8, dtype=np.float64)
    t = srv.submit_fit(x, y, ncomp=6, precision=64)
    srv.wait(t)
    got, _, _ = srv.wait(srv.submit_predict(t, xt, [2, 6]))
    ref = O.simpls_fit(x, y, ncomp=6)
    for j, k in enumerate([2, 6]):
        assert O.rel_err(got[j], O.simpls_predict(ref, xt, k)) < 1e-9
    srv.release(t)
    srv.close()


def test_server_rejects_oversized_and_unknown():
    srv = api.Server(budget_bytes=10**6, workers=1)
    x, y = W.latent_regression(500, 400, 2, 3, 0.4, 9, dtype=np.float32)
    with pytest.raises(api._lib.FastplsError, match="HBM budget"):
        srv.submit_fit(x, y, ncomp=2)
    with pytest.raises(Exception):
        srv.submit_predict(12345, x, [1])
    srv.close()


def test_predictions_queued_behind_their_fits():
    # predictions submitted before their model exists wait in the server's
    # queue (not on the client) and give the standalone results
    srv = api.Server(budget_bytes=150 * 10**9, workers=3)
    fits, preds = {}, {}
    for i, (method, n, p, q, a, cls) in enumerate(SPECS):
        x, y, lab = _data(i, method, n, p, q, cls)
        fits[i] = srv.submit_fit(x, y, labels=lab, classes=q if cls else None, ncomp=a,
                                 method=method, precision=32, **_kw(method, p))
        xt, _, _ = _data(70 + i, method, 29, p, q, False)
        preds[i] = srv.submit_predict(fits[i], xt, [a])
    for i, t in preds.items():
        got, _, _ = srv.wait(t)
        method, n, p, q, a, cls = SPECS[i]
        x, y, lab = _data(i, method, n, p, q, cls)
        xt, _, _ = _data(70 + i, method, 29, p, q, False)
        alone = api.fit_resident(x, y, labels=lab, classes=q if cls else None, ncomp=a,
                                 method=method, precision=32, **_kw(method, p))
        assert np.array_equal(got, alone.predict_path(xt, [a])), i
        alone.close()
    for t in fits.values():
        srv.wait(t)
        srv.release(t)
    srv.close()


def test_prediction_behind_a_failing_fit_reports_it():
    srv = api.Server(budget_bytes=150 * 10**9, workers=1)
    x = np.zeros((60, 12), dtype=np.float32)  # no spread: the fit fails on the device
    y = np.ones((60, 1), dtype=np.float32)
    t = srv.submit_fit(x, y, ncomp=2, method="simpls", precision=32)
    pt = srv.submit_predict(t, np.zeros((5, 12), dtype=np.float32), [1])
    with pytest.raises(Exception):
        srv.wait(t)
    with pytest.raises(Exception, match="fit failed|unknown model"):
        srv.wait(pt)
    srv.close()


def test_batched_fits_share_one_persistent_launch():
    """SIMPLS fits queued together (one worker, so later ones wait) run as
    batches in one persistent cooperative launch; every fit's predictions
    are bitwise those of the same fit made alone, and the oracle's."""
    srv = api.Server(workers=1)
    specs = [(200 + 37 * i, 150 + 61 * i, 1 + i % 4, 3 + i % 6) for i in range(16)]
    data, tickets = [], []
    for i, (n, p, q, a) in enumerate(specs):
        x, y = W.latent_regression(n, p, q, 4, 0.4, 300 + i, dtype=np.float32)
        data.append((x, y))
    # a larger fit first keeps the one worker busy while the small fits queue
    # up behind it (otherwise each small fit may finish before the next one
    # is submitted, and nothing is left to batch)
    xb, yb = W.latent_regression(6000, 12000, 3, 4, 0.4, 299, dtype=np.float32)
    blocker = srv.submit_fit(xb, yb, ncomp=40, precision=32)
    for i, (n, p, q, a) in enumerate(specs):
        x, y = data[i]
        tickets.append(srv.submit_fit(x, y, ncomp=a, precision=32))
    srv.wait(blocker)
    for t in tickets:
        srv.wait(t)
    stats = srv.batch_stats()
    assert stats["launches"] >= 1 and stats["fits"] >= 2, stats
    for i, (n, p, q, a) in enumerate(specs):
        x, y = data[i]
        xt, _ = W.latent_regression(23, p, q, 4, 0.4, 700 + i, dtype=np.float32)
        got, _, _ = srv.wait(srv.submit_predict(tickets[i], xt, [1, a]))
        alone = api.fit_resident(x, y, ncomp=a, precision=32)
        want = alone.predict_path(xt, [1, a])
        alone.close()
        assert np.array_equal(got, want), i
        ref = O.simpls_fit(x.astype(np.float64), y.astype(np.float64), ncomp=a)
        assert O.rel_err(got[1].astype(np.float64),
                         O.simpls_predict(ref, xt.astype(np.float64), a)) < 1e-5, i
        srv.release(tickets[i])
    srv.release(blocker)
    srv.close()
