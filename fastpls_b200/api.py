"""Python mirror of the fastPLS R API for the CUDA path (``backend = "cuda"``).

Names, arguments and defaults follow the reference's R functions
(R/main.R: pls 9746, predict.fastPLS 5206, pls.single.cv 10985;
R/native_api.R: has_cuda 601); the computation happens in
``libfastpls_b200.so`` through its C ABI. Matrices are numpy arrays with
rows = samples; they are handed to the library column-major.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib

SCALING = {"centering": 1, "autoscaling": 2, "none": 3}
METHODS = {"plssvd": 1, "simpls": 3, "opls": 4, "kernelpls": 5}
KERNELS = {"rbf": 2, "poly": 3}
METRICS = {"r2": 2, "q2": 3, "rmsd": 4}


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _mat(a, dtype):
    a = np.asarray(a, dtype=dtype)
    if a.ndim == 1:
        a = a[:, None]
    return np.asfortranarray(a)


def _dtype(precision):
    if precision not in (32, 64):
        raise ValueError("precision must be 32 or 64")
    return np.float32 if precision == 32 else np.float64


def to_bf16(a) -> np.ndarray:
    """BF16 bit patterns (uint16) of ``a``, rounded to nearest even from FP32.

    Predictors in precision 16 are handed to the library as these bits; a
    uint16 array is taken as bits already."""
    a = np.asarray(a)
    if a.dtype == np.uint16:
        return a
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    nan = (u & 0x7F800000) == 0x7F800000
    r = ((u + np.uint32(0x7FFF) + ((u >> 16) & np.uint32(1))) >> 16).astype(np.uint16)
    # NaN and infinity keep their class (truncation keeps the quiet bit set)
    return np.where(nan, (u >> 16).astype(np.uint16) | np.where((u & 0x7FFFFF) != 0, 0x40, 0).astype(np.uint16), r)


def from_bf16(bits) -> np.ndarray:
    """FP32 values of BF16 bit patterns."""
    b = np.ascontiguousarray(bits, dtype=np.uint16)
    return (b.astype(np.uint32) << 16).view(np.float32)


def _xmat(a, precision):
    """Predictor matrix in the storage type of ``precision`` (16 = BF16 bits)."""
    if precision == 16:
        b = to_bf16(a)
        if b.ndim == 1:
            b = b[:, None]
        return np.asfortranarray(b)
    return _mat(a, _dtype(precision))


def _odtype(precision):
    """Responses and results: FP32 for BF16 predictors."""
    return np.float32 if precision == 16 else _dtype(precision)


def has_cuda() -> bool:
    """True when a CUDA device is visible (has_cuda(), R/native_api.R:601)."""
    return _lib.load().fastpls_b200_device_count() > 0


def launch_count() -> int:
    return int(_lib.load().fastpls_b200_launch_count())


def encode_labels(y):
    """Factor-style encoding: sorted unique levels -> one-based codes."""
    levels, codes = np.unique(np.asarray(y), return_inverse=True)
    return (codes + 1).astype(np.int32), levels


@dataclass
class ResidentModel:
    """A model resident on the GPU (the R package's EXTPTR handle)."""

    handle: int
    precision: int
    n: int
    p: int
    q: int
    ncomp: int
    method: str
    classification: bool
    levels: np.ndarray | None = None
    feature_p: int = 0          # rows of R (p; n for kernel PLS)
    _freed: bool = field(default=False, repr=False)

    @property
    def dtype(self):
        """Type of responses and results (FP32 when predictors are BF16)."""
        return _odtype(self.precision)

    def _x(self, x):
        return _xmat(x, self.precision)

    def close(self):
        if not self._freed and self.handle:
            _lib.load().fastpls_resident_simpls_destroy(C.c_void_p(self.handle))
            self._freed = True

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- exports (fastpls_resident_export field ids) ----
    def export(self, field_id: int) -> np.ndarray:
        a, q, p, n = self.ncomp, self.q, self.p, self.n
        fp = self.feature_p or p
        shapes = {0: (fp, a), 1: (q, a), 2: (n, a), 3: (p,), 4: (p,), 5: (q,),
                  6: (fp, a), 7: (a + 1,)}
        shape = shapes[field_id]
        out = np.zeros(shape, dtype=self.dtype, order="F")
        err, cap = _lib.error_buffer()
        rc = _lib.load().fastpls_resident_export(
            C.c_void_p(self.handle), field_id, _p(out), out.size, err, cap)
        _lib.check(rc, err)
        return out

    def weights(self):
        return self.export(0)

    def loadings(self):
        return self.export(1)

    def scores(self):
        return self.export(2)

    def predict_path(self, x, prefixes, lda=False) -> np.ndarray:
        x = self._x(x)
        pre = np.ascontiguousarray(prefixes, dtype=np.int32)
        rows = x.shape[0]
        out = np.zeros(rows * self.q * len(pre), dtype=self.dtype)
        err, cap = _lib.error_buffer()
        rc = _lib.load().fastpls_resident_predict_path(
            C.c_void_p(self.handle), _p(x), rows, _p(pre), len(pre), int(lda),
            _p(out), err, cap)
        _lib.check(rc, err)
        return out.reshape((len(pre), self.q, rows)).transpose(0, 2, 1)

    def classify_path(self, x, prefixes, lda=False, top=1, responses=False):
        x = self._x(x)
        pre = np.ascontiguousarray(prefixes, dtype=np.int32)
        rows = x.shape[0]
        labels = np.zeros(rows * top * len(pre), dtype=np.int32)
        err, cap = _lib.error_buffer()
        if responses:
            resp = np.zeros(rows * self.q * len(pre), dtype=self.dtype)
            rc = _lib.load().fastpls_resident_classify_response_path(
                C.c_void_p(self.handle), _p(x), rows, _p(pre), len(pre),
                int(lda), top, _p(labels), _p(resp), err, cap)
        else:
            resp = None
            rc = _lib.load().fastpls_resident_classify_path(
                C.c_void_p(self.handle), _p(x), rows, _p(pre), len(pre),
                int(lda), top, _p(labels), err, cap)
        _lib.check(rc, err)
        lab = labels.reshape((len(pre), top, rows)).transpose(0, 2, 1)
        if responses:
            return lab, resp.reshape((len(pre), self.q, rows)).transpose(0, 2, 1)
        return lab

    def project(self, x, prefix):
        x = self._x(x)
        rows = x.shape[0]
        out = np.zeros((rows, prefix), dtype=self.dtype, order="F")
        err, cap = _lib.error_buffer()
        rc = _lib.load().fastpls_resident_project(
            C.c_void_p(self.handle), _p(x), rows, int(prefix), _p(out), err, cap)
        _lib.check(rc, err)
        return out

    def response_sums(self, x, y=None, labels=None, prefix=None):
        x = self._x(x)
        rows = x.shape[0]
        prefix = self.ncomp if prefix is None else prefix
        yy = None if y is None else _mat(y, self.dtype)
        lab = None if labels is None else np.ascontiguousarray(labels, dtype=np.int32)
        out = np.zeros(3 * self.q, dtype=self.dtype)
        err, cap = _lib.error_buffer()
        rc = _lib.load().fastpls_resident_response_sums(
            C.c_void_p(self.handle), _p(x), _p(yy), _p(lab), rows, int(prefix),
            _p(out), err, cap)
        _lib.check(rc, err)
        return out.reshape((self.q, 3))

    def vip(self):
        """Variable importance in projection (ViP()): an array of shape
        (q, ncomp, feature_p), entry [r, c, j] for response r and the
        component prefix 1..c+1."""
        fp = self.feature_p or self.p
        out = np.zeros(self.q * self.ncomp * fp)
        err, cap = _lib.error_buffer()
        rc = _lib.load().fastpls_b200_resident_vip(C.c_void_p(self.handle), _p(out), out.size,
                                                   err, cap)
        _lib.check(rc, err)
        return out.reshape((self.q, fp, self.ncomp)).transpose(0, 2, 1)

    def controls(self):
        vals = [C.c_int(0) for _ in range(6)]
        err, cap = _lib.error_buffer()
        rc = _lib.load().fastpls_resident_controls(
            C.c_void_p(self.handle), *[C.byref(v) for v in vals], err, cap)
        _lib.check(rc, err)
        keys = ["oversample", "power", "block", "block_limit",
                "implicit_operator", "predictor_crossprod_cache"]
        return {k: v.value for k, v in zip(keys, vals)}

    def compact(self, prepare_lda=False):
        err, cap = _lib.error_buffer()
        rc = _lib.load().fastpls_resident_compact(
            C.c_void_p(self.handle), int(prepare_lda), err, cap)
        _lib.check(rc, err)


def fit_resident(X, Y=None, labels=None, classes=None, ncomp=2,
                 scaling="centering", method="simpls", precision=64,
                 oversample=32, power=5, seed=1, retain_scores=True,
                 north=1, kernel="rbf", gamma=None, degree=3, coef0=1.0):
    """Fit one resident model through ``fastpls_resident_<method>_create``.

    ``precision`` 32 or 64 as in the reference; 16 stores the predictors as
    BF16 (``to_bf16``) with FP32 responses and results, all arithmetic FP64."""
    dt = _odtype(precision)
    x = _xmat(X, precision)
    n, p = x.shape
    lib = _lib.load()
    err, cap = _lib.error_buffer()
    if labels is not None:
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        q = int(classes if classes is not None else lab.max())
        y = None
    else:
        y = _mat(Y, dt)
        q = y.shape[1]
        lab = None
    sc = SCALING[scaling] if isinstance(scaling, str) else int(scaling)
    common = (_p(x), _p(y), _p(lab), precision, n, p, q, int(ncomp), sc,
              int(oversample), int(power), int(retain_scores), C.c_ulonglong(seed))
    if method == "simpls":
        h = lib.fastpls_resident_simpls_create(*common, err, cap)
    elif method == "plssvd":
        h = lib.fastpls_resident_plssvd_create(*common, err, cap)
    elif method == "opls":
        h = lib.fastpls_resident_opls_create(*common, int(north), err, cap)
    elif method == "kernelpls":
        g = float(gamma) if gamma is not None else 1.0 / p
        h = lib.fastpls_resident_kernelpls_create(
            *common, KERNELS[kernel], g, int(degree), float(coef0), err, cap)
    else:
        raise ValueError(f"unknown method {method!r}")
    if not h:
        raise _lib.FastplsError(err.value.decode(errors="replace"))
    feature_p = n if method == "kernelpls" else p
    return ResidentModel(handle=h, precision=precision, n=n, p=p, q=q,
                         ncomp=int(ncomp), method=method,
                         classification=labels is not None, feature_p=feature_p)


def export_model(model: ResidentModel, scores=True) -> dict:
    """The fields a SIMPLS / OPLS model needs to be rebuilt by
    ``import_model`` (export field ids 0, 1, 2, 3, 4, 5), as FP64 arrays."""
    out = {"method": model.method, "scaling": None, "classification": model.classification,
           "weights": model.export(0).astype(np.float64),
           "response_loadings": model.export(1).astype(np.float64),
           "mean_x": model.export(3).astype(np.float64),
           "scale_x": model.export(4).astype(np.float64),
           "mean_y": model.export(5).astype(np.float64)}
    if scores:
        out["scores"] = model.export(2).astype(np.float64)
    return out


def import_model(fields: dict, labels=None, precision=64, scaling="centering") -> ResidentModel:
    """Rebuild a resident SIMPLS / OPLS model from exported fields
    (``fastpls_b200_model_import``); ``labels`` (with ``fields["scores"]``)
    enable LDA on a classification model."""
    method = fields.get("method", "simpls")
    if method not in ("simpls", "opls"):
        raise ValueError("model import supports SIMPLS and OPLS models")
    R = np.asfortranarray(fields["weights"], dtype=np.float64)
    Qm = np.asfortranarray(fields["response_loadings"], dtype=np.float64)
    p, a = R.shape
    q = Qm.shape[0]
    T = fields.get("scores")
    T = None if T is None else np.asfortranarray(T, dtype=np.float64)
    n = 0 if T is None else T.shape[0]
    mx = np.ascontiguousarray(fields["mean_x"], dtype=np.float64)
    sx = np.ascontiguousarray(fields["scale_x"], dtype=np.float64)
    my = np.ascontiguousarray(fields["mean_y"], dtype=np.float64)
    lab = None if labels is None else np.ascontiguousarray(labels, dtype=np.int32)
    cls = bool(fields.get("classification", False) or labels is not None)
    sc = fields.get("scaling") or scaling
    sc = SCALING[sc] if isinstance(sc, str) else int(sc)
    err, cap = _lib.error_buffer()
    h = _lib.load().fastpls_b200_model_import(
        METHODS[method], precision, n, p, q, a, sc, int(cls), _p(R), _p(Qm), _p(T), _p(mx),
        _p(sx), _p(my), _p(lab), err, cap)
    if not h:
        raise _lib.FastplsError(err.value.decode(errors="replace"))
    return ResidentModel(handle=h, precision=precision, n=n, p=p, q=q, ncomp=a, method=method,
                         classification=cls, feature_p=p)


def cuda_gemm(left, right, precision=64):
    dt = _dtype(precision)
    a = _mat(left, dt)
    b = _mat(right, dt)
    out = np.zeros((a.shape[0], b.shape[1]), dtype=dt, order="F")
    err, cap = _lib.error_buffer()
    rc = _lib.load().fastpls_cuda_gemm(_p(a), _p(b), precision, a.shape[0],
                                       a.shape[1], b.shape[1], _p(out), err, cap)
    _lib.check(rc, err)
    return out


def cv_regression(X, Y, folds, prefixes, scaling="centering", method="simpls",
                  metric="q2", precision=64, store_predictions=False,
                  oversample=32, power=5, seed=1):
    """``fastpls_resident_{simpls,plssvd}_cv_regression``."""
    dt = _dtype(precision)
    x = _mat(X, dt)
    y = _mat(Y, dt)
    n, p = x.shape
    q = y.shape[1]
    folds = np.ascontiguousarray(folds, dtype=np.int32)
    pre = np.ascontiguousarray(prefixes, dtype=np.int32)
    k = len(pre)
    nf = int(folds.max()) if folds.size else 0
    status = np.zeros(max(nf, 1), dtype=np.int32)
    metrics, q2, rmsd, r2 = (np.zeros(k) for _ in range(4))
    preds = np.zeros(k * n * q) if store_predictions else None
    sc = SCALING[scaling] if isinstance(scaling, str) else int(scaling)
    fn = {"simpls": "fastpls_resident_simpls_cv_regression",
          "plssvd": "fastpls_resident_plssvd_cv_regression"}[method]
    err, cap = _lib.error_buffer()
    rc = getattr(_lib.load(), fn)(
        _p(x), _p(y), _p(folds), precision, n, p, q, _p(pre), k, sc,
        METRICS[metric] if isinstance(metric, str) else int(metric),
        int(oversample), int(power), C.c_ulonglong(seed), int(store_predictions),
        _p(preds), _p(status), _p(metrics), _p(q2), _p(rmsd), _p(r2), err, cap)
    _lib.check(rc, err)
    out = dict(metrics=metrics, q2=q2, rmsd=rmsd, observed_r2=r2, status=status,
               predictions=None)
    if preds is not None:
        out["predictions"] = preds.reshape((k, q, n)).transpose(0, 2, 1)
    return out


def cv_classification(X, labels, classes, folds, prefixes, scaling="centering",
                      method="simpls", lda=False, precision=64,
                      store_predictions=False, store_scores=False,
                      oversample=32, power=5, seed=1):
    """``fastpls_resident_{simpls,plssvd}_cv_classification``."""
    dt = _dtype(precision)
    x = _mat(X, dt)
    n, p = x.shape
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    folds = np.ascontiguousarray(folds, dtype=np.int32)
    pre = np.ascontiguousarray(prefixes, dtype=np.int32)
    k = len(pre)
    nf = int(folds.max()) if folds.size else 0
    status = np.zeros(max(nf, 1), dtype=np.int32)
    metrics = np.zeros(k)
    preds = np.zeros(n * k, dtype=np.int32) if store_predictions else None
    scores = np.zeros(n * int(classes) * k, dtype=dt) if store_scores else None
    sc = SCALING[scaling] if isinstance(scaling, str) else int(scaling)
    fn = {"simpls": "fastpls_resident_simpls_cv_classification",
          "plssvd": "fastpls_resident_plssvd_cv_classification"}[method]
    err, cap = _lib.error_buffer()
    rc = getattr(_lib.load(), fn)(
        _p(x), _p(lab), _p(folds), precision, n, p, int(classes), _p(pre), k, sc,
        int(lda), int(oversample), int(power), C.c_ulonglong(seed),
        int(store_predictions), int(store_scores), _p(preds), _p(scores),
        _p(status), _p(metrics), err, cap)
    _lib.check(rc, err)
    out = dict(metrics=metrics, status=status, predictions=None, scores=None)
    if preds is not None:
        out["predictions"] = preds.reshape((k, n)).T
    if scores is not None:
        out["scores"] = scores.reshape((k, int(classes), n)).transpose(0, 2, 1)
    return out


def set_product_digits(digits: int) -> None:
    """int8 digits per FP64 value in the batched engine's products with the
    shared Gram (0 = FP64 DMMA GEMMs); process-wide."""
    _lib.load().fastpls_b200_set_product_digits(int(digits))


def product_digits() -> int:
    return int(_lib.load().fastpls_b200_product_digits())


def set_batch_lanes(lanes: int) -> None:
    """Stream lanes of the batched engine (1..4); process-wide."""
    _lib.load().fastpls_b200_set_batch_lanes(int(lanes))


def batch_lanes() -> int:
    return int(_lib.load().fastpls_b200_batch_lanes())


def set_argmax_guard(margin: float) -> None:
    """Relative top-two score margin under which the batched classification
    engine refits an instance with FP64 products (0 disables); process-wide."""
    _lib.load().fastpls_b200_set_argmax_guard(float(margin))


def argmax_guard() -> float:
    return float(_lib.load().fastpls_b200_argmax_guard())


def set_persistent(enable: bool) -> None:
    """Single-fit SIMPLS component loop as one persistent launch (default)
    or as the per-kernel loop; process-wide."""
    _lib.load().fastpls_b200_set_persistent(1 if enable else 0)


def persistent() -> bool:
    return bool(_lib.load().fastpls_b200_persistent())


def set_autotune(enable: bool) -> None:
    """Autotuning of the batched engine's group schedule (lanes x tile
    width); process-wide, on by default."""
    _lib.load().fastpls_b200_set_autotune(1 if enable else 0)


def autotune() -> bool:
    return bool(_lib.load().fastpls_b200_autotune())


def batched_stats() -> dict:
    """Schedule statistics of the last batched call."""
    vals = [C.c_int(0) for _ in range(6)]
    _lib.load().fastpls_b200_batched_stats(*[C.byref(v) for v in vals])
    keys = ("groups", "graph_replays", "graph_captures", "tuned", "lanes", "tile_n")
    return {k: v.value for k, v in zip(keys, vals)}


def last_fit_times() -> dict:
    """Device milliseconds of this thread's last resident fit: the input
    copies and the fit proper."""
    a, b = C.c_double(0), C.c_double(0)
    _lib.load().fastpls_b200_last_fit_times(C.byref(a), C.byref(b))
    return {"copy_ms": a.value, "fit_ms": b.value}


def release_workspace() -> None:
    """Free the batched engine's persistent device workspace."""
    _lib.load().fastpls_b200_release_workspace()


def guard_refits() -> int:
    """Instances refitted with FP64 products by the last batched
    classification call."""
    return int(_lib.load().fastpls_b200_guard_refits())


def int8_crossprod(a, b=None, digits=6, tile_n=0, pair=-1):
    """a^T b (b = None: a^T a, symmetric) by the int8 split product on the
    tensor cores; a is k x m, b is k x n (FP64). tile_n: 128, 192, 256 or 0
    (chosen for the shape); pair: 1 = CTA-pair 256-row tiles, 0 or -1 =
    single-CTA tiles (-1: automatic)."""
    A = _mat(a, np.float64)
    sym = b is None
    B = A if sym else _mat(b, np.float64)
    if A.shape[0] != B.shape[0]:
        raise ValueError("a and b need the same number of rows")
    k, m = A.shape
    n = B.shape[1]
    out = np.zeros((m, n), order="F")
    err, cap = _lib.error_buffer()
    rc = _lib.load().fastpls_b200_int8_crossprod(
        _p(A), max(k, 1), _p(B), max(k, 1), m, n, k, int(digits), 1 if sym else 0,
        int(tile_n), int(pair), _p(out), m, err, cap)
    _lib.check(rc, err)
    return out


def cv_permutation(X, Y, folds, permutations, prefixes, scaling="centering",
                   metric="q2", precision=32, digits=None):
    """Batched CV over the observed responses and their row permutations
    (``fastpls_b200_simpls_cv_permutation``). Returns arrays of shape
    (permutations + 1, prefixes), row 0 the observed responses. digits
    selects the product precision for this call (None: the process setting,
    see set_product_digits)."""
    if digits is not None:
        old = product_digits()
        set_product_digits(digits)
        try:
            return cv_permutation(X, Y, folds, permutations, prefixes, scaling,
                                  metric, precision, None)
        finally:
            set_product_digits(old)
    dt = _dtype(precision)
    x = _mat(X, dt)
    y = _mat(Y, dt)
    n, p = x.shape
    q = y.shape[1]
    folds = np.ascontiguousarray(folds, dtype=np.int32)
    perms = None
    P = 0
    if permutations is not None and len(permutations):
        perms = np.ascontiguousarray(permutations, dtype=np.int32)
        P = perms.shape[0]
    pre = np.ascontiguousarray(prefixes, dtype=np.int32)
    k = len(pre)
    metrics, q2, rmsd, r2 = (np.zeros((P + 1) * k) for _ in range(4))
    status = np.zeros(int(folds.max()), dtype=np.int32)
    sc = SCALING[scaling] if isinstance(scaling, str) else int(scaling)
    err, cap = _lib.error_buffer()
    rc = _lib.load().fastpls_b200_simpls_cv_permutation(
        _p(x), _p(y), _p(folds), _p(perms), P, precision, n, p, q, _p(pre), k,
        sc, METRICS[metric] if isinstance(metric, str) else int(metric),
        _p(metrics), _p(q2), _p(rmsd), _p(r2), _p(status), err, cap)
    _lib.check(rc, err)
    shape = (P + 1, k)
    return dict(metrics=metrics.reshape(shape), q2=q2.reshape(shape),
                rmsd=rmsd.reshape(shape), observed_r2=r2.reshape(shape),
                status=status)


def fastcor(a, b=None, byrow=True, diag=True, precision=64):
    """Pearson correlations between the rows (byrow) or columns of a and b
    (fastcor(), R/main.R:12799). Without b the full a-by-a matrix."""
    dt = _dtype(precision)
    A = _mat(a, dt)
    B = None if b is None else _mat(b, dt)
    ua = A.shape[0] if byrow else A.shape[1]
    if B is None:
        out = np.zeros((ua, ua), order="F")
    else:
        ub = B.shape[0] if byrow else B.shape[1]
        out = np.zeros(ua) if (diag and ua == ub) else np.zeros((ua, ub), order="F")
    err, cap = _lib.error_buffer()
    rc = _lib.load().fastpls_b200_fastcor(
        _p(A), _p(B), precision, A.shape[0], A.shape[1],
        0 if B is None else B.shape[0], 0 if B is None else B.shape[1],
        int(byrow), int(diag), _p(out), err, cap)
    _lib.check(rc, err)
    return out


AUDIT_FIELDS = ("certified", "deterministic_fallback", "attempts", "effective_oversample",
                "effective_power", "effective_seed", "subspace_error",
                "singular_value_error", "triplet_residual", "omitted_direction_ratio")


def fastsvd(x, ncomp, oversample=32, power=5, seed=1, precision=64, audit=False):
    """Truncated SVD on the device with the audited rSVD policy
    (fastsvd(backend = "cuda")): u, d, v (and the audit record as a dict
    when ``audit``)."""
    dt = _dtype(precision)
    X = _mat(x, dt)
    n, p = X.shape
    k = int(ncomp)
    u = np.zeros((n, k), order="F")
    v = np.zeros((p, k), order="F")
    d = np.zeros(k)
    rec = np.zeros(10)
    err, cap = _lib.error_buffer()
    rc = _lib.load().fastpls_b200_fastsvd_audited(
        _p(X), precision, n, p, k, int(oversample), int(power), C.c_ulonglong(seed), _p(u),
        _p(d), _p(v), _p(rec), err, cap)
    _lib.check(rc, err)
    if audit:
        info = dict(zip(AUDIT_FIELDS, rec.tolist()))
        for key in ("certified", "deterministic_fallback"):
            info[key] = bool(info[key])
        for key in ("attempts", "effective_oversample", "effective_power", "effective_seed"):
            info[key] = int(info[key])
        return u, d, v, info
    return u, d, v


def cv_permutation_classification(X, labels, classes, folds, permutations, prefixes,
                                  scaling="centering", precision=32, digits=None, lda=False):
    """Batched classification CV over the observed labels and their row
    permutations (``fastpls_b200_simpls_cv_permutation_classification_head``;
    argmax head, or LDA on the latent scores with lda=True). Returns
    dict(accuracy=(permutations + 1, prefixes), status)."""
    if digits is not None:
        old = product_digits()
        set_product_digits(digits)
        try:
            return cv_permutation_classification(X, labels, classes, folds, permutations,
                                                 prefixes, scaling, precision, None, lda)
        finally:
            set_product_digits(old)
    dt = _dtype(precision)
    x = _mat(X, dt)
    n, p = x.shape
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    folds = np.ascontiguousarray(folds, dtype=np.int32)
    perms = None
    P = 0
    if permutations is not None and len(permutations):
        perms = np.ascontiguousarray(permutations, dtype=np.int32)
        P = perms.shape[0]
    pre = np.ascontiguousarray(prefixes, dtype=np.int32)
    k = len(pre)
    acc = np.zeros((P + 1) * k)
    status = np.zeros(int(folds.max()), dtype=np.int32)
    sc = SCALING[scaling] if isinstance(scaling, str) else int(scaling)
    err, cap = _lib.error_buffer()
    rc = _lib.load().fastpls_b200_simpls_cv_permutation_classification_head(
        _p(x), _p(lab), _p(folds), _p(perms), P, precision, n, p, int(classes), _p(pre), k, sc,
        1 if lda else 0, _p(acc), _p(status), err, cap)
    _lib.check(rc, err)
    return dict(accuracy=acc.reshape((P + 1, k)), status=status)


class Server:
    """Serving loop on the device (fastpls_b200_server_*): continuous
    admission of fit and predict requests by HBM footprint, resident models,
    merged predictions per model. Fit tickets double as model ids.

    borrow=True (default) submits inputs without a host copy: the server
    reads the arrays in place, and this object keeps a reference to each
    request's arrays until its wait() has returned (or close())."""

    def __init__(self, budget_bytes=150 * 10**9, workers=4, borrow=True):
        err, cap = _lib.error_buffer()
        self._lib = _lib.load()
        self._h = self._lib.fastpls_b200_server_create(int(budget_bytes), int(workers), err, cap)
        if not self._h:
            raise _lib.FastplsError(err.value.decode())
        self._models = {}
        self._pending = {}
        self._held = {}
        self._borrow = bool(borrow)
        self._lib.fastpls_b200_server_set_borrow(self._h, 1 if self._borrow else 0)

    def submit_fit(self, X, Y=None, labels=None, classes=None, ncomp=2,
                   method="simpls", scaling="centering", precision=32, north=1,
                   kernel="rbf", gamma=None, degree=3, coef0=1.0):
        dt = _dtype(precision)
        x = _mat(X, dt)
        n, p = x.shape
        if labels is not None:
            lab = np.ascontiguousarray(labels, dtype=np.int32)
            q = int(classes if classes is not None else lab.max())
            y = None
        else:
            y = _mat(Y, dt)
            q = y.shape[1]
            lab = None
        g = float(gamma) if gamma is not None else 1.0 / p
        t = C.c_ulonglong(0)
        err, cap = _lib.error_buffer()
        rc = self._lib.fastpls_b200_server_submit_fit(
            self._h, METHODS[method], _p(x), _p(y), _p(lab), precision, n, p, q,
            int(ncomp), SCALING[scaling] if isinstance(scaling, str) else int(scaling),
            int(north), KERNELS.get(kernel, 2), g, int(degree), float(coef0),
            C.byref(t), err, cap)
        _lib.check(rc, err)
        self._models[t.value] = (q, precision, p)
        if self._borrow:
            self._held[t.value] = (x, y, lab)
        return t.value

    def submit_predict(self, model, X, prefixes, lda=False):
        q, precision, p = self._models[model]
        x = _mat(X, _dtype(precision))
        pre = np.ascontiguousarray(prefixes, dtype=np.int32)
        t = C.c_ulonglong(0)
        err, cap = _lib.error_buffer()
        rc = self._lib.fastpls_b200_server_submit_predict(
            self._h, C.c_ulonglong(model), _p(x), x.shape[0], x.shape[1], precision,
            _p(pre), len(pre), int(lda), C.byref(t), err, cap)
        _lib.check(rc, err)
        self._pending[t.value] = (x.shape[0], q, len(pre), precision)
        if self._borrow:
            self._held[t.value] = (x,)
        return t.value

    def wait(self, ticket, timeout=600.0):
        """(result, queue_ms, service_ms); result is the prediction array
        (prefixes x rows x q) for predict tickets, the model id for fits."""
        qms, sms = C.c_double(0), C.c_double(0)
        err, cap = _lib.error_buffer()
        if ticket in self._pending:
            rows, q, k, precision = self._pending.pop(ticket)
            out = np.zeros(rows * q * k, dtype=_dtype(precision))
            rc = self._lib.fastpls_b200_server_wait(
                self._h, C.c_ulonglong(ticket), float(timeout), _p(out), out.nbytes,
                C.byref(qms), C.byref(sms), err, cap)
            _lib.check(rc, err)
            self._held.pop(ticket, None)  # the request has finished reading x
            return out.reshape((k, q, rows)).transpose(0, 2, 1), qms.value, sms.value
        rc = self._lib.fastpls_b200_server_wait(
            self._h, C.c_ulonglong(ticket), float(timeout), None, 0,
            C.byref(qms), C.byref(sms), err, cap)
        _lib.check(rc, err)
        self._held.pop(ticket, None)
        return ticket, qms.value, sms.value

    def release(self, model):
        err, cap = _lib.error_buffer()
        _lib.check(self._lib.fastpls_b200_server_release(self._h, C.c_ulonglong(model), err, cap), err)
        self._models.pop(model, None)

    def stats(self):
        a, b, c = C.c_size_t(0), C.c_size_t(0), C.c_size_t(0)
        self._lib.fastpls_b200_server_stats(self._h, C.byref(a), C.byref(b), C.byref(c))
        return dict(bytes_in_use=a.value, queued=b.value, resident_models=c.value)

    def batch_stats(self):
        """Persistent launches that carried batches of fits, and those fits."""
        a, b = C.c_size_t(0), C.c_size_t(0)
        self._lib.fastpls_b200_server_batch_stats(self._h, C.byref(a), C.byref(b))
        return dict(launches=a.value, fits=b.value)

    def close(self):
        if self._h:
            self._lib.fastpls_b200_server_destroy(self._h)
            self._h = None
        self._held = {}  # no worker reads borrowed inputs any more

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
