"""CPU oracle for the fastPLS model-fitting path -- TEST INFRASTRUCTURE ONLY.

A plain numpy FP64 restatement of the reference's CPU algorithms. Only
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of
``bench.py`` may import it, and only as the checker. The product library never
calls it (there is no CPU fallback in ``fastpls_b200``).

Parity is pinned two ways (see tests/test_oracle_pins.py):
  * against the known answers in the reference's own C++ tests
    (core/tests/test_core_plssvd.cpp:89-90, test_core_simpls.cpp:84-117,
    test_core_lda.cpp), restated as fixtures in tests/golden/;
  * against the reference core itself, compiled from its headers into
    oracle/_ref/libfastpls_ref.so (oracle/Makefile), on seeded inputs.

Dominant directions.  The reference obtains each SIMPLS direction and the
PLS-SVD factors from a randomized SVD whose sketch width is
``min(k + oversample, min(p, m))``
(inst/include/fastpls/core/simpls.hpp:237-243, rsvd.hpp:191-200). Whenever that
width equals ``min(p, m)`` the sketch spans the whole response space and the
result is the exact singular subspace, independent of the random draws; the
reference itself then takes the dense-SVD branch (rsvd.hpp:197-200). The oracle
computes the exact SVD, so signs of singular vectors are arbitrary and callers
align them (``align_signs``).

Conventions: matrices are column-major in the C ABI but plain 2-D arrays here
(rows = samples); labels are one-based; scaling 1 = centre, 2 = autoscale
(sd with n-1), 3 = none (inst/include/fastpls/core/classification.hpp:18-22).
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "column_statistics", "simpls_fit", "simpls_block_size", "simpls_predict", "simpls_project",
    "plssvd_fit", "plssvd_predict", "lda_train", "lda_discriminants",
    "row_argmax", "topk", "response_sums", "cv_regression", "opls_fit",
    "opls_predict", "kernelpls_fit", "kernelpls_predict",
    "cv_classification", "permutation_pvalue", "align_signs", "rel_err",
    "fastcor", "vip",
]


# --------------------------------------------------------------------------
# preprocessing
# --------------------------------------------------------------------------
def column_statistics(x: np.ndarray, scaling: int):
    """Column centre and scale (supervised.hpp:53-90).

    Centre = mean unless scaling == 3. Scale = sd with n-1 computed from the
    raw sum of squares, clamped at 0, replaced by 1 when not finite or <= 0;
    only for scaling == 2.
    """
    x = np.asarray(x, dtype=np.float64)
    n, p = x.shape
    centre = np.zeros(p)
    scale = np.ones(p)
    if scaling != 3:
        s = x.sum(axis=0)
        ss = (x * x).sum(axis=0)
        centre = s / n
        if scaling == 2:
            centred = np.maximum(0.0, ss - n * centre * centre)
            with np.errstate(invalid="ignore", divide="ignore"):
                sd = np.sqrt(centred / max(n - 1, 1))
            bad = ~np.isfinite(sd) | (sd <= 0)
            sd[bad] = 1.0
            scale = sd
    return centre, scale


def _one_hot(labels, classes):
    labels = np.asarray(labels, dtype=np.int64)
    y = np.zeros((labels.size, classes))
    y[np.arange(labels.size), labels - 1] = 1.0
    return y


def _prepare(x, y, labels, classes, scaling):
    """Scaled predictors, centred cross-product and response means.

    Dense responses: supervised.hpp:27-124 (S = Xs^T Y - colsum(Xs) mean(Y)^T).
    Labels: classification.hpp:88-186 (S = class sums - total * prior), which
    equals Xs^T (onehot - prior); response mean = class priors.
    """
    x = np.asarray(x, dtype=np.float64)
    centre, scale = column_statistics(x, scaling)
    xs = (x - centre) / scale
    if labels is not None:
        yd = _one_hot(labels, classes)
    else:
        yd = np.asarray(y, dtype=np.float64)
        if yd.ndim == 1:
            yd = yd[:, None]
    ymean = yd.mean(axis=0)
    s = xs.T @ yd - np.outer(xs.sum(axis=0), ymean)
    return xs, s, centre, scale, ymean, yd


# --------------------------------------------------------------------------
# SIMPLS
# --------------------------------------------------------------------------
def _dominant_left(s: np.ndarray) -> np.ndarray:
    """Unit dominant left singular vector of s (refresh_directions,
    simpls.hpp:226-368, exact-span case)."""
    u, _, _ = np.linalg.svd(s, full_matrices=False)
    return u[:, 0].copy()


def simpls_block_size(n, p, q, components, classification, fp32=False):
    """Candidate directions taken from one decomposition of S.

    Rule of the CUDA resident SIMPLS (src/cuda_resident_simpls.cuh:144-153):
    classification with q <= 2048 classes, components >= 4 and n p q >= 5e8
    -> min(64, components, p, q); FP32 regression whose p x q cross-covariance
    exceeds 512 MiB and components >= 4 -> min(8, components, p, q); else 1.
    The R/CPU path (simpls_candidate_block_size, simpls.hpp:43-62, called with
    a maximum of 64 at src/r_api.cpp:1155) gives the same classification
    blocks; its regression blocks start at p q > 64 Mi elements instead.
    """
    work = float(n) * float(p) * float(q)
    cap = min(int(components), int(p), int(q))
    if classification and q <= 2048 and components >= 4 and work >= 5.0e8:
        return max(1, min(64, cap))
    if (not classification and fp32 and components >= 4
            and float(p) * float(q) * 4.0 > 512.0 * 1024.0 * 1024.0):
        return max(1, min(8, cap))
    return 1


def simpls_fit(x, y=None, labels=None, classes=None, ncomp=2, scaling=1,
               reorthogonalize=False, block=None, classification=None):
    """Sequential SIMPLS (fit_simpls_preprocessed, simpls.hpp:479-763).

    Directions come in candidate blocks (simpls.hpp:547-567): at the start of
    a block of ``use`` components the leading ``use`` left singular vectors of
    the deflated cross-product S are computed once, and component j of the
    block takes candidate j as its r (simpls.hpp:588-595). ``block`` defaults
    to ``simpls_block_size`` (1 outside large classification fits, which is
    the per-component dominant direction).
    Per component (simpls.hpp:588-756): t = Xs r; r, t /= ||t||;
    p = Xs^T t; q = S0^T r; v = p - V (V^T p) (twice when reorthogonalize);
    v /= ||v||; S -= v (v^T S). The FP64 CPU path runs with
    reorthogonalize = False (src/r_api.cpp:1179 and :1408-1411).
    Returns a dict with R (p x a), Q (m x a), V (p x a), T (n x a),
    centre, scale, ymean.
    """
    xs, s0, centre, scale, ymean, _ = _prepare(x, y, labels, classes, scaling)
    n, p = xs.shape
    m = s0.shape[1]
    a = min(int(ncomp), p, max(n - 1, 1))
    if classification is None:
        classification = labels is not None
    if block is None:
        block = simpls_block_size(n, p, m, a, classification)
    R = np.zeros((p, a))
    Q = np.zeros((m, a))
    V = np.zeros((p, a))
    T = np.zeros((n, a))
    s = s0.copy()
    done = 0
    k = 0
    stopped = False
    while k < a and not stopped:
        use = max(1, min(int(block), a - k, p, m))
        u, _, _ = np.linalg.svd(s, full_matrices=False)
        candidates = u[:, :use].copy()
        for j in range(use):
            r = candidates[:, j].copy()
            t = xs @ r
            if reorthogonalize and k > 0:
                for _ in range(2):
                    proj = T[:, :k].T @ t
                    t = t - T[:, :k] @ proj
                    r = r - R[:, :k] @ proj
            tn = np.linalg.norm(t)
            if not np.isfinite(tn) or tn <= 0:
                stopped = True
                break
            t = t / tn
            r = r / tn
            ld = xs.T @ t
            q = s0.T @ r
            v = ld.copy()
            for _ in range(2 if reorthogonalize else 1):
                if k:
                    v = v - V[:, :k] @ (V[:, :k].T @ v)
            vn = np.linalg.norm(v)
            if not np.isfinite(vn) or vn <= 0:
                stopped = True
                break
            v = v / vn
            s = s - np.outer(v, v @ s)
            R[:, k], Q[:, k], V[:, k], T[:, k] = r, q, v, t
            k += 1
            done = k
    return dict(R=R[:, :done], Q=Q[:, :done], V=V[:, :done], T=T[:, :done],
                centre=centre, scale=scale, ymean=ymean)


def simpls_project(model, x, prefix):
    """Test scores Xs R[:, :prefix] (project_scores, cross_validation.hpp:947-963)."""
    xs = (np.asarray(x, dtype=np.float64) - model["centre"]) / model["scale"]
    return xs @ model["R"][:, :prefix]


def simpls_predict(model, x, prefix):
    """Yhat = ymean + Xs R_a Q_a^T (predict_simpls_preprocessed,
    simpls.hpp:1049-1076)."""
    t = simpls_project(model, x, prefix)
    return model["ymean"] + t @ model["Q"][:, :prefix].T


# --------------------------------------------------------------------------
# PLS-SVD
# --------------------------------------------------------------------------
def plssvd_fit(x, y=None, labels=None, classes=None, prefixes=(2,), scaling=1):
    """PLS-SVD (assemble_plssvd_model, plssvd.hpp:57-166).

    SVD of the centred cross-product S (p x m); R = U_k; T = Xs R;
    G = T^T T; for each prefix j: W_j = chol-solve(G_j, diag(sigma_1..j))
    V_j^T, so Yhat = ymean + T_j W_j.
    """
    xs, s, centre, scale, ymean, _ = _prepare(x, y, labels, classes, scaling)
    prefixes = [int(v) for v in prefixes]
    k = max(prefixes)
    if k > min(s.shape):
        raise ValueError("fastPLS PLS-SVD component count exceeds cross-covariance rank")
    u, sig, vt = np.linalg.svd(s, full_matrices=False)
    R = u[:, :k].copy()
    Qv = vt[:k].T.copy()
    T = xs @ R
    G = T.T @ T
    W = []
    for j in prefixes:
        lat = np.linalg.solve(G[:j, :j], np.diag(sig[:j]))
        W.append(lat @ Qv[:, :j].T)
    return dict(R=R, Q=Qv, T=T, sigma=sig[:k].copy(), W=W, prefixes=prefixes,
                centre=centre, scale=scale, ymean=ymean)


def plssvd_predict(model, x, prefix_index):
    """Yhat = ymean + Xs R_j W_j (predict_plssvd_from_scores,
    cross_validation.hpp:965-994)."""
    j = model["prefixes"][prefix_index]
    xs = (np.asarray(x, dtype=np.float64) - model["centre"]) / model["scale"]
    return model["ymean"] + (xs @ model["R"][:, :j]) @ model["W"][prefix_index]


# --------------------------------------------------------------------------
# OPLS and kernel PLS
# --------------------------------------------------------------------------
def opls_fit(x, y=None, labels=None, classes=None, ncomp=2, scaling=1, north=1):
    """OPLS filters + SIMPLS (opls.hpp:120-290, oplspls.hpp:30-74).

    Each filter on the standardised Xf: w = unit dominant left singular
    vector of Xf^T Yc; t = Xf w; p = Xf^T t / t't; w_o = normalise(p -
    (w'p / w'w) w); t_o = Xf w_o; p_o = Xf^T t_o / t_o't_o; Xf -= t_o p_o^T.
    The predictive SIMPLS runs on the filtered Xf (no further scaling).
    Returns the SIMPLS dict plus Wo, Po and R_eff (weights acting on the
    standardised, unfiltered predictors).
    """
    xs, _, centre, scale, ymean, yd = _prepare(x, y, labels, classes, scaling)
    yc = yd - ymean
    xf = xs.copy()
    p = xf.shape[1]
    Wo, Po = [], []
    for _ in range(int(north)):
        w = _dominant_left(xf.T @ yc)
        w = w / np.linalg.norm(w)
        t = xf @ w
        pl = xf.T @ t / (t @ t)
        wo = pl - (w @ pl) / (w @ w) * w
        wo = wo / np.linalg.norm(wo)
        to = xf @ wo
        po = xf.T @ to / (to @ to)
        xf = xf - np.outer(to, po)
        Wo.append(wo)
        Po.append(po)
    inner = simpls_fit(xf, yd, ncomp=ncomp, scaling=3,
                       classification=labels is not None)
    R = inner["R"].copy()
    for wo, po in zip(reversed(Wo), reversed(Po)):
        R = R - np.outer(wo, R.T @ po)
    inner.update(R_eff=R, Wo=Wo, Po=Po, centre=centre, scale=scale)
    return inner


def opls_predict(model, x, prefix):
    xs = (np.asarray(x, dtype=np.float64) - model["centre"]) / model["scale"]
    return model["ymean"] + (xs @ model["R_eff"][:, :prefix]) @ model["Q"][:, :prefix].T


def _kernel(a, b, kind, gamma, degree, coef0):
    dots = a @ b.T
    if kind == 2:  # RBF (kernels.hpp:41-55)
        na = (a * a).sum(axis=1)[:, None]
        nb = (b * b).sum(axis=1)[None, :]
        d = np.maximum(na + nb - 2.0 * dots, 0.0)
        return np.exp(-gamma * d)
    return (gamma * dots + coef0) ** degree  # polynomial (kernels.hpp:29-35)


def kernelpls_fit(x, y=None, labels=None, classes=None, ncomp=2, scaling=1,
                  kind=2, gamma=1.0, degree=3, coef0=1.0):
    """Kernel PLS (kernelpls.hpp:85-196): K = phi(Xs Xs^T) double-centred
    with its column means and grand mean, then SIMPLS on K."""
    xs, _, centre, scale, ymean, yd = _prepare(x, y, labels, classes, scaling)
    K = _kernel(xs, xs, kind, gamma, degree, coef0)
    cm = K.mean(axis=0)
    g = cm.mean()
    Kc = K - cm[:, None] - cm[None, :] + g
    inner = simpls_fit(Kc, yd, ncomp=ncomp, scaling=3,
                       classification=labels is not None)
    inner.update(reference=xs, kcol=cm, kgrand=g, kind=kind, gamma=gamma,
                 degree=degree, coef0=coef0, centre=centre, scale=scale)
    return inner


def kernelpls_predict(model, x, prefix):
    xs = (np.asarray(x, dtype=np.float64) - model["centre"]) / model["scale"]
    Kt = _kernel(xs, model["reference"], model["kind"], model["gamma"],
                 model["degree"], model["coef0"])
    Kt = Kt - Kt.mean(axis=1)[:, None] - model["kcol"][None, :] + model["kgrand"]
    return model["ymean"] + (Kt @ model["R"][:, :prefix]) @ model["Q"][:, :prefix].T


# --------------------------------------------------------------------------
# LDA on latent scores
# --------------------------------------------------------------------------
_RIDGE_GRID = (1e-8, 1e-6, 1e-5, 1e-4, 1e-3, 1e-2)


def _chol_solve(cov, means, ridge):
    """lda_cholesky_solve (lda.hpp:33-83): Cholesky of cov + ridge I, then
    two triangular solves per class; fails on a non-positive pivot."""
    k = cov.shape[0]
    L = np.zeros((k, k))
    for i in range(k):
        for j in range(i + 1):
            v = cov[i, j] + (ridge if i == j else 0.0) - L[i, :j] @ L[j, :j]
            if i == j:
                if not np.isfinite(v) or v <= 0:
                    return None
                L[i, i] = np.sqrt(v)
            else:
                L[i, j] = v / L[j, j]
    sol = np.zeros((k, means.shape[0]))
    for c in range(means.shape[0]):
        z = np.zeros(k)
        for i in range(k):
            z[i] = (means[c, i] - L[i, :i] @ z[:i]) / L[i, i]
        w = np.zeros(k)
        for i in range(k - 1, -1, -1):
            w[i] = (z[i] - L[i + 1:, i] @ w[i + 1:]) / L[i, i]
            if not np.isfinite(w[i]):
                return None
        sol[:, c] = w
    return sol.T


def lda_train(scores, labels, classes, prefixes):
    """Pooled-covariance LDA per prefix (train_lda_prefixes, lda.hpp:156-223;
    finalize_lda_prefixes, lda.hpp:88-153).

    Class means; pooled = (T^T T - sum_c n_c mu_c mu_c^T) / max(1, n - c);
    ridge = rho * trace/k for rho in 1e-8,1e-6,...,1e-2 (first that factors);
    linear = Sigma^-1 mu_c; constant = -0.5 mu_c^T linear + log(prior).
    """
    scores = np.asarray(scores, dtype=np.float64)
    labels = np.asarray(labels, dtype=np.int64)
    n = scores.shape[0]
    kmax = max(prefixes)
    counts = np.bincount(labels - 1, minlength=classes).astype(np.float64)
    if np.any(counts <= 0):
        raise ValueError("fastPLS LDA received an empty class")
    means = np.zeros((classes, kmax))
    for c in range(classes):
        means[c] = scores[labels == c + 1, :kmax].sum(axis=0) / counts[c]
    gram = scores[:, :kmax].T @ scores[:, :kmax]
    pooled = gram - (means.T * counts) @ means
    pooled /= max(1, n - classes if n > classes else 1)
    models = []
    for k in prefixes:
        cov = pooled[:k, :k]
        sc = np.trace(cov) / k
        if not np.isfinite(sc) or sc <= 0:
            sc = 1.0
        lin = None
        for rho in _RIDGE_GRID:
            lin = _chol_solve(cov, means[:, :k], rho * sc)
            if lin is not None:
                ridge = rho * sc
                break
        if lin is None:
            raise RuntimeError("fastPLS LDA Cholesky factorization failed for every regularization level")
        priors = counts / n
        const = -0.5 * np.einsum("ck,ck->c", means[:, :k], lin) + np.log(
            np.maximum(priors, np.finfo(np.float64).tiny))
        models.append(dict(linear=lin, constants=const, ridge=ridge, k=k))
    return models


def lda_discriminants(model, scores):
    """constants + scores_k linear^T (lda_scores, lda.hpp:284-305)."""
    k = model["k"]
    return model["constants"] + np.asarray(scores)[:, :k] @ model["linear"].T


def row_argmax(values):
    """One-based argmax per row; the first maximal column wins
    (row_argmax, classification.hpp:401-425; resident_topk uses strict >)."""
    return np.argmax(np.asarray(values), axis=1).astype(np.int32) + 1


def topk(values, top):
    """One-based top-k classes per row, ties resolved toward the lower index
    (resident_topk_one_pass, src/cuda_resident_api.cuh:29-53)."""
    values = np.asarray(values)
    order = np.argsort(-values, axis=1, kind="stable")
    return (order[:, :top] + 1).astype(np.int32)


# --------------------------------------------------------------------------
# metrics and cross-validation
# --------------------------------------------------------------------------
def response_sums(pred, y, training_mean):
    """Per response: SSE, SS about the training mean, SS about the observed
    mean (response_sums, src/cuda_resident_metrics.cuh:9-43)."""
    y = np.asarray(y, dtype=np.float64)
    pred = np.asarray(pred, dtype=np.float64)
    out = np.zeros((y.shape[1], 3))
    out[:, 0] = ((y - pred) ** 2).sum(axis=0)
    out[:, 1] = ((y - training_mean) ** 2).sum(axis=0)
    out[:, 2] = ((y - y.mean(axis=0)) ** 2).sum(axis=0)
    return out


def _partitions(folds):
    """fold_partitions (cross_validation.hpp:772-798): fold 0 rows are always
    training rows, never tested."""
    folds = np.asarray(folds)
    k = int(folds.max())
    out = []
    for f in range(1, k + 1):
        test = np.nonzero(folds == f)[0]
        train = np.nonzero((folds != f) & (folds != 0))[0]
        out.append((train, test))
    return out


def cv_regression(x, y, folds, prefixes, scaling=1, family=3, metric=3,
                  store_predictions=False):
    """Regression CV (cross_validate_regression, cross_validation.hpp:1790-2173).

    Per fold: fit on the training rows with training-row preprocessing, predict
    the held-out rows for every prefix, accumulate SSE; Q2 = 1 - SSE / sum over
    folds of held-out SS about the training mean; RMSD = sqrt(SSE / count);
    R2 = 1 - SSE / total SS of y. ``metric`` picks 2 = R2, 3 = Q2, 4 = RMSD.
    """
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    if y.ndim == 1:
        y = y[:, None]
    n, m = y.shape
    prefixes = [int(v) for v in prefixes]
    parts = _partitions(folds)
    sse = np.zeros(len(prefixes))
    counts = np.zeros(len(prefixes))
    fold_ss = 0.0
    status = np.zeros(len(parts), dtype=np.int32)
    preds = np.zeros((len(prefixes), n, m)) if store_predictions else None
    total_ss = float(((y - y.mean(axis=0)) ** 2).sum())
    for f, (train, test) in enumerate(parts):
        if test.size == 0:
            status[f] = 2
            continue
        if family == 3:
            model = simpls_fit(x[train], y[train], ncomp=max(prefixes),
                               scaling=scaling)
        else:
            model = plssvd_fit(x[train], y[train], prefixes=prefixes,
                               scaling=scaling)
        fold_ss += float(((y[test] - model["ymean"]) ** 2).sum())
        for j, a in enumerate(prefixes):
            if family == 3:
                yh = simpls_predict(model, x[test], a)
            else:
                yh = plssvd_predict(model, x[test], j)
            sse[j] += float(((y[test] - yh) ** 2).sum())
            counts[j] += yh.size
            if preds is not None:
                preds[j][test] = yh
        status[f] = 1
    with np.errstate(invalid="ignore", divide="ignore"):
        rmsd = np.where(counts > 0, np.sqrt(sse / np.maximum(counts, 1)), np.nan)
    q2 = 1.0 - sse / fold_ss if fold_ss > 0 else np.full(len(prefixes), np.nan)
    r2 = 1.0 - sse / total_ss if total_ss > 0 else np.full(len(prefixes), np.nan)
    metrics = {2: r2, 3: q2, 4: rmsd}[metric]
    return dict(metrics=metrics, q2=q2, rmsd=rmsd, observed_r2=r2, sse=sse,
                status=status, predictions=preds)


def cv_classification(x, labels, classes, folds, prefixes, scaling=1, family=3,
                      head=0, store_predictions=False):
    """Classification CV accuracy (cross_validate_classification,
    cross_validation.hpp:1360-1788; the CUDA driver
    src/cuda_resident_api.cuh:538-768 has the same fold semantics).

    Classes absent from a fold's training rows are dropped and the remaining
    ones compacted; a fold with <= 1 active class predicts that class
    (status 4). head 0 = argmax of Yhat, 1 = LDA on the latent scores.
    """
    x = np.asarray(x, dtype=np.float64)
    labels = np.asarray(labels, dtype=np.int64)
    n = labels.size
    prefixes = [int(v) for v in prefixes]
    parts = _partitions(folds)
    correct = np.zeros(len(prefixes))
    total = np.zeros(len(prefixes))
    status = np.zeros(len(parts), dtype=np.int32)
    preds = np.zeros((n, len(prefixes)), dtype=np.int32) if store_predictions else None
    for f, (train, test) in enumerate(parts):
        if test.size == 0:
            status[f] = 2
            continue
        present = np.unique(labels[train])
        if present.size <= 1:
            fallback = int(present[0]) if present.size else 1
            for j in range(len(prefixes)):
                correct[j] += np.sum(labels[test] == fallback)
                total[j] += test.size
                if preds is not None:
                    preds[test, j] = fallback
            status[f] = 4
            continue
        remap = np.zeros(classes + 1, dtype=np.int64)
        remap[present] = np.arange(1, present.size + 1)
        compact = remap[labels[train]]
        c = present.size
        if family == 3:
            model = simpls_fit(x[train], labels=compact, classes=c,
                               ncomp=max(prefixes), scaling=scaling)
            ttrain = model["T"]
            ttest = simpls_project(model, x[test], max(prefixes))
        else:
            model = plssvd_fit(x[train], labels=compact, classes=c,
                               prefixes=prefixes, scaling=scaling)
            ttrain = model["T"]
            xs = (x[test] - model["centre"]) / model["scale"]
            ttest = xs @ model["R"]
        ldas = lda_train(ttrain, compact, c, prefixes) if head == 1 else None
        for j, a in enumerate(prefixes):
            if head == 1:
                d = lda_discriminants(ldas[j], ttest)
            elif family == 3:
                d = model["ymean"] + ttest[:, :a] @ model["Q"][:, :a].T
            else:
                d = model["ymean"] + ttest[:, :a] @ model["W"][j]
            pred = present[row_argmax(d) - 1]
            correct[j] += np.sum(pred == labels[test])
            total[j] += test.size
            if preds is not None:
                preds[test, j] = pred
        status[f] = 1
    metrics = np.where(total > 0, correct / np.maximum(total, 1), np.nan)
    return dict(metrics=metrics, status=status, predictions=preds)


def fastcor(a, b=None, byrow=True, diag=True):
    """Pearson correlations (fastcor_values / normalized_units,
    src/r_api.cpp:4054-4166): each unit (row when byrow) centred and scaled
    to unit norm, NaN when non-finite or of zero spread; L R^T, or paired
    dot products when diag (only with b and matching unit counts)."""
    def units(x):
        x = np.asarray(x, dtype=np.float64)
        u = x if byrow else x.T
        mean = u.mean(axis=1, keepdims=True)
        c = u - mean
        norm = np.sqrt((c * c).sum(axis=1, keepdims=True))
        ok = np.all(np.isfinite(u), axis=1, keepdims=True) & (norm > 0)
        with np.errstate(invalid="ignore", divide="ignore"):
            return np.where(ok, c / norm, np.nan)
    L = units(a)
    if b is None:
        return L @ L.T
    R = units(b)
    if diag and L.shape[0] == R.shape[0]:
        return (L * R).sum(axis=1)
    return L @ R.T


def permutation_pvalue(permuted, observed, lower_tail=False):
    """(b + 1) / (B + 1) over finite permuted values
    (.fastpls_permutation_pvalue, R/main.R:2702-2718)."""
    permuted = np.asarray(permuted, dtype=np.float64)
    valid = np.isfinite(permuted)
    done = int(valid.sum())
    if not done or not np.isfinite(observed):
        return float("nan")
    if lower_tail:
        extreme = int(np.sum(permuted[valid] <= observed))
    else:
        extreme = int(np.sum(permuted[valid] >= observed))
    return (extreme + 1) / (done + 1)


# --------------------------------------------------------------------------
# comparison helpers
# --------------------------------------------------------------------------
def vip(R, Q, T):
    """Variable importance in projection (vip_values, src/r_api.cpp:3973-4025):
    array (q, a, p); entry [r, c, j] = sqrt(p * sum_{c'<=c} (R_jc'^2 /
    ||R_c'||^2) SS_c' / sum_{c'<=c} SS_c') with SS_c = Q_rc^2 ||T_c||^2."""
    R = np.asarray(R, dtype=np.float64)
    Q = np.asarray(Q, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    p, a = R.shape
    tss = (T * T).sum(axis=0)
    wss = (R * R).sum(axis=0)
    wn = np.where(wss > 0, R * R / np.where(wss > 0, wss, 1.0), 0.0)   # p x a
    out = np.empty((Q.shape[0], a, p))
    for r in range(Q.shape[0]):
        expl = Q[r] ** 2 * tss                     # a
        den = np.cumsum(expl)
        num = np.cumsum(wn * expl, axis=1)         # p x a
        with np.errstate(invalid="ignore", divide="ignore"):
            val = np.sqrt(p * num / den)
        val[:, den <= 0] = np.nan
        out[r] = val.T
    return out


def align_signs(test, ref):
    """Flip columns of ``test`` so each has a non-negative inner product with
    the matching column of ``ref`` (singular-vector sign alignment)."""
    test = np.array(test, dtype=np.float64, copy=True)
    ref = np.asarray(ref, dtype=np.float64)
    if test.ndim == 1:
        return test if float(test @ ref) >= 0 else -test
    for j in range(test.shape[1]):
        if float(test[:, j] @ ref[:, j]) < 0:
            test[:, j] = -test[:, j]
    return test


def rel_err(test, ref):
    """Frobenius relative error ||test - ref|| / ||ref||."""
    test = np.asarray(test, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.linalg.norm(ref)
    num = np.linalg.norm(test - ref)
    return float(num / den) if den > 0 else float(num)
