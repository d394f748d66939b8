"""ctypes access to the compiled reference core -- TEST INFRASTRUCTURE ONLY.

``oracle/_ref/libfastpls_ref.so`` is the reference's own header-only FP64
numerics (fastPLS inst/include/fastpls/core) compiled by ``oracle/Makefile``
with a project-written OpenBLAS backend adapter (``oracle/ref_harness.cpp``).
It validates the numpy restatement in ``oracle/pls_oracle.py`` and is the CPU
baseline that ``bench.py`` times. Arrays are passed column-major (Fortran
order), as the reference's C ABI expects.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libfastpls_ref.so")
_lib = None

_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="F_CONTIGUOUS")
_I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build(reference_root=None):
    """Compile the reference core harness (needs the reference tree, found at
    ``reference_root`` or the FASTPLS_REFERENCE_ROOT environment variable)."""
    if reference_root is None:
        reference_root = os.environ.get("FASTPLS_REFERENCE_ROOT", "/root/reference")
    subprocess.run(["make", "-s", f"REF={reference_root}"], cwd=_HERE,
                   check=True)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(
                f"{LIB_PATH} is missing; build it with `make -C oracle`")
        _lib = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        _lib.ref_simpls_fit.restype = C.c_int
        _lib.ref_plssvd_fit.restype = C.c_int
        _lib.ref_cv_regression.restype = C.c_int
        _lib.ref_cv_classification.restype = C.c_int
        _lib.ref_lda.restype = C.c_int
        del vp
    return _lib


def set_threads(n: int):
    lib().ref_set_threads(C.c_int(int(n)))


def _f(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _err():
    return C.create_string_buffer(512)


def simpls_fit(x, y=None, labels=None, classes=None, ncomp=2, scaling=1,
               oversample=32, power=5, seed=1):
    x = _f(x)
    n, p = x.shape
    if labels is not None:
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        m = int(classes)
        yy = None
    else:
        yy = _f(y if np.ndim(y) == 2 else np.asarray(y)[:, None])
        lab = None
        m = yy.shape[1]
    a = min(int(ncomp), p, max(n - 1, 1))
    R = np.zeros((p, a), order="F")
    Q = np.zeros((m, a), order="F")
    V = np.zeros((p, a), order="F")
    T = np.zeros((n, a), order="F")
    cx, sx, my = np.zeros(p), np.zeros(p), np.zeros(m)
    done = C.c_int(0)
    secs = C.c_double(0)
    err = _err()
    rc = lib().ref_simpls_fit(
        _ptr(x), _ptr(yy), _ptr(lab), n, p, m, int(ncomp), int(scaling),
        int(oversample), int(power), C.c_uint(seed), _ptr(R), _ptr(Q),
        _ptr(V), _ptr(T), _ptr(cx), _ptr(sx), _ptr(my), C.byref(done),
        C.byref(secs), err, C.c_size_t(512))
    if rc:
        raise RuntimeError(err.value.decode())
    k = done.value
    return dict(R=R[:, :k], Q=Q[:, :k], V=V[:, :k], T=T[:, :k], centre=cx,
                scale=sx, ymean=my, seconds=secs.value)


def plssvd_fit(x, y=None, labels=None, classes=None, prefixes=(2,),
               scaling=1, oversample=32, power=5, seed=1):
    x = _f(x)
    n, p = x.shape
    if labels is not None:
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        m = int(classes)
        yy = None
    else:
        yy = _f(y if np.ndim(y) == 2 else np.asarray(y)[:, None])
        lab = None
        m = yy.shape[1]
    pre = np.ascontiguousarray(prefixes, dtype=np.int32)
    k = int(pre.max())
    R = np.zeros((p, k), order="F")
    Q = np.zeros((m, k), order="F")
    T = np.zeros((n, k), order="F")
    sig = np.zeros(k)
    W = np.zeros(int(pre.sum()) * m)
    cx, sx, my = np.zeros(p), np.zeros(p), np.zeros(m)
    err = _err()
    rc = lib().ref_plssvd_fit(
        _ptr(x), _ptr(yy), _ptr(lab), n, p, m, _ptr(pre), len(pre),
        int(scaling), int(oversample), int(power), C.c_uint(seed), _ptr(R),
        _ptr(Q), _ptr(T), _ptr(sig), _ptr(W), _ptr(cx), _ptr(sx), _ptr(my),
        err, C.c_size_t(512))
    if rc:
        raise RuntimeError(err.value.decode())
    ws, off = [], 0
    for j in pre:
        ws.append(W[off:off + j * m].reshape((j, m), order="F"))
        off += j * m
    return dict(R=R, Q=Q, T=T, sigma=sig, W=ws, prefixes=[int(v) for v in pre],
                centre=cx, scale=sx, ymean=my)


def cv_regression(x, y, folds, prefixes, scaling=1, family=3, metric=3,
                  oversample=32, power=5, seed=1, store_predictions=False):
    x = _f(x)
    y = _f(y if np.ndim(y) == 2 else np.asarray(y)[:, None])
    n, p = x.shape
    m = y.shape[1]
    folds = np.ascontiguousarray(folds, dtype=np.int32)
    pre = np.ascontiguousarray(prefixes, dtype=np.int32)
    k = len(pre)
    nf = int(folds.max())
    status = np.zeros(nf, dtype=np.int32)
    metrics, q2, rmsd, r2 = (np.zeros(k) for _ in range(4))
    preds = np.zeros(k * n * m) if store_predictions else None
    err = _err()
    rc = lib().ref_cv_regression(
        _ptr(x), _ptr(y), _ptr(folds), n, p, m, _ptr(pre), k, int(scaling),
        int(family), int(metric), int(oversample), int(power), C.c_uint(seed),
        _ptr(preds), _ptr(status), _ptr(metrics), _ptr(q2), _ptr(rmsd),
        _ptr(r2), err, C.c_size_t(512))
    if rc:
        raise RuntimeError(err.value.decode())
    out = dict(metrics=metrics, q2=q2, rmsd=rmsd, observed_r2=r2,
               status=status, predictions=None)
    if preds is not None:
        out["predictions"] = preds.reshape((k, m, n)).transpose(0, 2, 1)
    return out


def cv_classification(x, labels, classes, folds, prefixes, scaling=1,
                      family=3, head=0, oversample=32, power=5, seed=1,
                      store_predictions=False):
    x = _f(x)
    n, p = x.shape
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    folds = np.ascontiguousarray(folds, dtype=np.int32)
    pre = np.ascontiguousarray(prefixes, dtype=np.int32)
    k = len(pre)
    nf = int(folds.max())
    status = np.zeros(nf, dtype=np.int32)
    metrics = np.zeros(k)
    preds = np.zeros(n * k, dtype=np.int32) if store_predictions else None
    err = _err()
    rc = lib().ref_cv_classification(
        _ptr(x), _ptr(lab), _ptr(folds), n, p, int(classes), _ptr(pre), k,
        int(scaling), int(family), int(head), int(oversample), int(power),
        C.c_uint(seed), _ptr(preds), _ptr(status), _ptr(metrics), err,
        C.c_size_t(512))
    if rc:
        raise RuntimeError(err.value.decode())
    out = dict(metrics=metrics, status=status, predictions=None)
    if preds is not None:
        out["predictions"] = preds.reshape((k, n)).T
    return out


def lda(train_scores, labels, classes, prefixes, test_scores):
    ts = _f(train_scores)
    te = _f(test_scores)
    n, a = ts.shape
    rows = te.shape[0]
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    pre = np.ascontiguousarray(prefixes, dtype=np.int32)
    k = len(pre)
    disc = np.zeros(k * rows * int(classes))
    pred = np.zeros(k * rows, dtype=np.int32)
    err = _err()
    rc = lib().ref_lda(_ptr(ts), _ptr(lab), n, a, int(classes), _ptr(pre), k,
                       _ptr(te), rows, _ptr(disc), _ptr(pred), err,
                       C.c_size_t(512))
    if rc:
        raise RuntimeError(err.value.decode())
    return (disc.reshape((k, int(classes), rows)).transpose(0, 2, 1),
            pred.reshape((k, rows)).T)


def opls_predict(x, y, ncomp, north, scaling, xtest):
    x, xt = _f(x), _f(xtest)
    y = _f(y if np.ndim(y) == 2 else np.asarray(y)[:, None])
    n, p = x.shape
    m = y.shape[1]
    out = np.zeros((xt.shape[0], m), order="F")
    err = _err()
    rc = lib().ref_opls_predict(_ptr(x), _ptr(y), n, p, m, int(ncomp), int(north),
                                int(scaling), _ptr(xt), xt.shape[0], _ptr(out),
                                err, C.c_size_t(512))
    if rc:
        raise RuntimeError(err.value.decode())
    return out


def kernelpls_predict(x, y, ncomp, scaling, kind, gamma, degree, coef0, xtest):
    x, xt = _f(x), _f(xtest)
    y = _f(y if np.ndim(y) == 2 else np.asarray(y)[:, None])
    n, p = x.shape
    m = y.shape[1]
    out = np.zeros((xt.shape[0], m), order="F")
    err = _err()
    rc = lib().ref_kernelpls_predict(_ptr(x), _ptr(y), n, p, m, int(ncomp),
                                     int(scaling), int(kind), C.c_double(gamma),
                                     int(degree), C.c_double(coef0), _ptr(xt),
                                     xt.shape[0], _ptr(out), err, C.c_size_t(512))
    if rc:
        raise RuntimeError(err.value.decode())
    return out
