"""The C ABI library: loads, exports every declared symbol, and rejects bad
arguments with the reference's messages before touching the device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from fastpls_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fastpls_b200.h")


def declared():
    text = open(HEADER).read()
    return re.findall(r"FASTPLS_B200_API\s+[\w\s\*]+?\b(fastpls_\w+)\s*\(", text)


def test_header_declares_reference_abi():
    names = set(declared())
    reference = {
        "fastpls_cuda_gemm", "fastpls_resident_simpls_cv_classification",
        "fastpls_resident_simpls_cv_regression",
        "fastpls_resident_plssvd_cv_classification",
        "fastpls_resident_plssvd_cv_regression", "fastpls_resident_simpls_create",
        "fastpls_resident_plssvd_create", "fastpls_resident_opls_create",
        "fastpls_resident_kernelpls_create", "fastpls_resident_predict_path",
        "fastpls_resident_simpls_destroy", "fastpls_resident_export",
        "fastpls_resident_classify_path",
        "fastpls_resident_classify_response_path",
        "fastpls_resident_response_sums", "fastpls_resident_project",
        "fastpls_resident_controls", "fastpls_resident_compact"}
    assert reference <= names


def test_library_exports_every_declared_symbol(lib):
    for name in declared():
        assert hasattr(lib, name), name
    assert set(declared()) == set(_lib.SIGNATURES)


def _err():
    return C.create_string_buffer(256), C.c_size_t(256)


def test_create_rejects_bad_precision(lib):
    x = np.zeros((4, 3))
    err, cap = _err()
    h = lib.fastpls_resident_simpls_create(
        x.ctypes.data_as(C.c_void_p), None, None, 8, 4, 3, 1, 1, 1, 32, 5, 1,
        C.c_ulonglong(1), err, cap)
    assert not h and err.value == b"invalid resident matrix or precision"
    h = lib.fastpls_resident_simpls_create(
        x.ctypes.data_as(C.c_void_p), None, None, 64, 4, 3, 1, 1, 1, 32, 5, 7,
        C.c_ulonglong(1), err, cap)
    assert not h and err.value == b"invalid resident score-retention request"


def test_gemm_and_null_model_errors(lib):
    err, cap = _err()
    assert lib.fastpls_cuda_gemm(None, None, 64, 1, 1, 1, None, err, cap) == 1
    assert err.value == b"invalid CUDA matrix multiplication input"
    assert lib.fastpls_resident_export(None, 0, None, 0, err, cap) == 1
    assert err.value == b"null resident model"
    assert lib.fastpls_resident_compact(None, 0, err, cap) == 1
    assert err.value == b"invalid resident compaction request"
    assert lib.fastpls_resident_predict_path(None, None, 1, None, 1, 0, None, err, cap) == 1
    assert err.value == b"invalid resident prediction-path model"


def test_cv_control_validation(lib):
    err, cap = _err()
    rc = lib.fastpls_resident_simpls_cv_regression(
        None, None, None, 16, 10, 3, 1, None, 1, 1, 3, 32, 5, C.c_ulonglong(1), 0,
        None, None, None, None, None, None, err, cap)
    assert rc == 1 and err.value == b"invalid resident CUDA regression CV controls"
    rc = lib.fastpls_resident_simpls_cv_classification(
        None, None, None, 32, 10, 3, 2, None, 1, 1, 5, 32, 5, C.c_ulonglong(1), 0, 0,
        None, None, None, None, err, cap)
    assert rc == 1 and err.value == b"invalid resident CUDA CV controls"


def test_error_buffer_truncates_safely(lib):
    err = C.create_string_buffer(8)
    assert lib.fastpls_cuda_gemm(None, None, 64, 1, 1, 1, None, err, C.c_size_t(8)) == 1
    assert err.value == b"invalid"


def test_device_count_without_gpu_is_nonnegative(lib):
    assert lib.fastpls_b200_device_count() >= 0


def _reference_header():
    root = os.environ.get("FASTPLS_REFERENCE_ROOT", "/root/reference")
    path = os.path.join(root, "src", "cuda_resident_api.h")
    return path if os.path.exists(path) else None


@pytest.mark.parametrize("lang,compiler", [("c++", "g++"), ("c", "gcc")])
def test_header_compiles_together_with_reference_header(tmp_path, lang, compiler):
    """One translation unit includes the reference's C ABI header
    (src/cuda_resident_api.h) and this library's header: a function whose
    name matches but whose signature differs is a conflicting extern "C"
    redeclaration and fails the compile. Each reference entry point is also
    bound to a pointer of the reference's type through this header's
    declaration."""
    import shutil
    import subprocess

    ref = _reference_header()
    if ref is None:
        pytest.skip("reference tree not present (set FASTPLS_REFERENCE_ROOT)")
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not found")
    names = re.findall(r"\b(fastpls_\w+)\s*\(", open(ref).read())
    assert len(names) == 18
    body = "\n".join(f"__typeof__({n}) *p_{n} = &{n};" for n in names)
    src = tmp_path / ("abi." + ("cpp" if lang == "c++" else "c"))
    src.write_text(f'#include "{ref}"\n#include "{HEADER}"\n{body}\n')
    proc = subprocess.run([compiler, "-x", lang, "-fsyntax-only", "-Wall", "-Werror", str(src)],
                          capture_output=True, text=True)
    assert proc.returncode == 0, proc.stderr
