"""Exact CPU emulation of the library's int8 split product -- TEST
INFRASTRUCTURE ONLY.

The reference forms every product of the fitting path in FP64 BLAS
(inst/include/fastpls/core/linalg.hpp via its BLAS backend). The B200 library
can instead run the products with the shared Gram of the batched CV engine on
the int8 tensor cores by splitting each FP64 value into signed 8-bit digits.
This module restates that split operation for operation, so the device result
can be checked bit for bit (the integer digit products are exact on both
sides; the FP64 epilogue is reproduced in the same order):

  * row scale 2^e with e from frexp(max |row|) (2^e > max |row|);
  * v0 = (x 2^-e) 127, d_s = rint(v_s), v_{s+1} = (v_s - d_s) 254;
  * diagonals d = s + t <= digits - 1, in passes of four diagonals (tile
    width 128) or two (widths 192 and 256); within a pass v = sum over d
    from high to low of w_d acc_d, w_d = 1/(127^2 254^d), acc_d the exact
    integer sum of the digit-pair products;
  * each pass adds (v 2^e_a) 2^e_b to the result; k is split into segments of
    at most floor((2^31 - 1) / (127^2 digits) / 64) * 64 so that int32 sums
    stay exact.

Accuracy against the FP64 product is checked separately (tests), and the
batched engine that uses it is checked against the FP64 oracle of the
reference's algorithm within the 1e-5 relative tolerance.
"""
from __future__ import annotations

import numpy as np

PASS = 4
KB = 64


def split(rows, digits):
    """rows (R x K) FP64 -> (planes: list of R x K integer-valued float64,
    scale: R powers of two)."""
    rows = np.asarray(rows, dtype=np.float64)
    R, K = rows.shape
    mx = np.max(np.abs(rows), axis=1) if K else np.zeros(R)
    ok = (mx > 0) & np.isfinite(mx)
    _, e = np.frexp(np.where(ok, mx, 1.0))
    inv = np.where(ok, np.ldexp(1.0, -e), 0.0)
    scale = np.where(ok, np.ldexp(1.0, e), 1.0)
    v = (rows * inv[:, None]) * 127.0
    planes = []
    for _ in range(digits):
        r = np.rint(v)
        planes.append(r)
        v = (v - r) * 254.0
    return planes, scale


def weights(digits):
    return [1.0 / (16129.0 * 254.0 ** d) for d in range(digits)]


def pass_diagonals(tile_n):
    return 4 if tile_n == 128 else 2


def product(a_rows, b_rows, digits, per_pass=PASS):
    """C = A B^T for A (M x K), B (N x K), as the device computes it with
    `per_pass` diagonals combined per pass."""
    A, sa = split(a_rows, digits)
    B, sb = split(b_rows, digits)
    M, K = np.shape(a_rows)
    N = np.shape(b_rows)[0]
    w = weights(digits)
    seg = max(1, (2147483647 // (16129 * digits)) // KB) * KB
    kp = max(KB, -(-K // KB) * KB)
    C = None
    for k0 in range(0, kp, seg):
        k1 = min(K, k0 + seg)
        for lo in range(0, digits, per_pass):
            hi = min(digits - 1, lo + per_pass - 1)
            v = np.zeros((M, N))
            for d in range(hi, lo - 1, -1):
                acc = np.zeros((M, N))
                for s in range(d + 1):
                    if k1 > k0:
                        acc += A[s][:, k0:k1] @ B[d - s][:, k0:k1].T
                v = v + w[d] * acc
            val = (v * sa[:, None]) * sb[None, :]
            C = val if C is None else C + val
    return C


def error_bound(a_rows, b_rows, digits):
    """Bound on |product - A B^T| per element: the neglected digit tail of
    each operand (1/2 of the last digit) and the dropped diagonals,
    relative to max|a_i| max|b_j| K, with FP64 rounding slack."""
    a = np.abs(np.asarray(a_rows, dtype=np.float64))
    b = np.abs(np.asarray(b_rows, dtype=np.float64))
    K = a.shape[1]
    ma = a.max(axis=1) if K else np.zeros(a.shape[0])
    mb = b.max(axis=1) if K else np.zeros(b.shape[0])
    unit = 2.0 ** -(7.99 * digits - 1.0) * (digits + 2)
    return (unit + 1e-15) * 4.0 * np.outer(ma, mb) * max(K, 1)
