"""Seeded synthetic inputs with the shapes of the benchmark configurations.

The reference ships no benchmark data for this path; inputs follow the latent
factor model X = T W^T diag(scale) + noise (column-centred), Y = T C + noise.
Draws use numpy's Philox counter-based generator keyed by (seed, stream id),
so every array is reproducible from its seed and stream id alone.
"""
from __future__ import annotations

import numpy as np

STREAM_T, STREAM_W, STREAM_NOISE, STREAM_C, STREAM_YNOISE, STREAM_SCALE = range(6)
STREAM_FOLDS, STREAM_PERM = 16, 17


def rng(seed: int, stream: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(key=[int(seed), int(stream)]))


def latent_regression(n, p, m, k, noise, seed, ynoise=0.1, sigma=None,
                      log_normal_scales=False, dtype=np.float32):
    """X (n x p, column-centred) and Y (n x m), both Fortran-ordered."""
    t = rng(seed, STREAM_T).standard_normal((n, k))
    w = rng(seed, STREAM_W).standard_normal((p, k))
    if sigma is not None:
        t = t * np.asarray(sigma)[None, :]
    x = t @ w.T
    if log_normal_scales:
        x *= np.exp(rng(seed, STREAM_SCALE).standard_normal(p))[None, :]
    x += noise * rng(seed, STREAM_NOISE).standard_normal((n, p))
    x -= x.mean(axis=0, keepdims=True)
    c = rng(seed, STREAM_C).standard_normal((k, m))
    y = t @ c + ynoise * rng(seed, STREAM_YNOISE).standard_normal((n, m))
    return np.asfortranarray(x.astype(dtype)), np.asfortranarray(y.astype(dtype))


def latent_classification(n, p, classes, k, noise, seed, sigma=None,
                          dtype=np.float32):
    """X (n x p, column-centred) and one-based labels = argmax(T C)."""
    t = rng(seed, STREAM_T).standard_normal((n, k))
    if sigma is not None:
        t = t * np.asarray(sigma)[None, :]
    w = rng(seed, STREAM_W).standard_normal((p, k))
    x = t @ w.T + noise * rng(seed, STREAM_NOISE).standard_normal((n, p))
    x -= x.mean(axis=0, keepdims=True)
    c = rng(seed, STREAM_C).standard_normal((k, classes))
    labels = np.argmax(t @ c, axis=1).astype(np.int32) + 1
    return np.asfortranarray(x.astype(dtype)), labels


def uneven_folds(n, k, seed, low=None, high=None):
    """One-based fold vector of a seeded shuffle with uneven fold sizes.

    Sizes are drawn in [low, high] (default: +-4% around n/k) and adjusted to
    sum to n; rows are assigned by a seeded permutation.
    """
    g = rng(seed, STREAM_FOLDS)
    base = n // k
    low = low if low is not None else int(base * 0.96)
    high = high if high is not None else int(np.ceil(base * 1.04))
    while True:
        sizes = g.integers(low, high + 1, size=k)
        diff = n - int(sizes.sum())
        i = 0
        while diff != 0 and i < 100000:
            j = i % k
            if diff > 0 and sizes[j] < high:
                sizes[j] += 1
                diff -= 1
            elif diff < 0 and sizes[j] > low:
                sizes[j] -= 1
                diff += 1
            i += 1
        if diff == 0:
            break
    folds = np.repeat(np.arange(1, k + 1, dtype=np.int32), sizes)
    return folds[g.permutation(n)].astype(np.int32)


def permutations(n, count, seed):
    """``count`` seeded row permutations (0-based int32, one per row)."""
    g = rng(seed, STREAM_PERM)
    if count <= 0:
        return np.zeros((0, n), dtype=np.int32)
    return np.stack([g.permutation(n).astype(np.int32) for _ in range(count)])


# Named workloads (sizes from the benchmark configurations).
def config_plain_simpls(dtype=np.float64):
    """500 x 2000, m = 3, k = 5, noise 0.5, Y noise 0.1, seed 1, ncomp 10."""
    return latent_regression(500, 2000, 3, 5, 0.5, 1, dtype=dtype)


def config_cv_permutation(n=5000, p=10000, dtype=np.float32):
    """5000 x 10000, k = 10, noise 0.3, m = 3, 10 uneven folds, 200 perms."""
    x, y = latent_regression(n, p, 3, 10, 0.3, 3, dtype=dtype)
    folds = uneven_folds(n, 10, 3)
    return x, y, folds


# ---------------------------------------------------------------------------
# Full-size configurations, drawn on the device (torch's CUDA Philox
# generator, seeded) because the host generator is far slower at these sizes.
# The same host arrays then feed the device fit and the FP64 reference.

def mixed_precision_config(seed=4, n=100_000, p=20_000, m=10, k=50, noise=0.5):
    """The mixed-precision SIMPLS configuration: X = T W^T diag(s) + noise
    (n x p, column-centred, column scales s ~ logN(0, 1)), rounded to BF16;
    Y = T C + 0.1 noise (n x m). Returns (bits, y): bits the BF16 bit
    patterns of X as an n x p Fortran-ordered uint16 array, y float32 n x m
    Fortran-ordered."""
    import torch

    dev = torch.device("cuda")
    g = torch.Generator(device=dev).manual_seed(seed)
    t = torch.randn(n, k, generator=g, device=dev)
    w = torch.randn(p, k, generator=g, device=dev)
    scale = torch.exp(torch.randn(p, generator=g, device=dev))
    c = torch.randn(k, m, generator=g, device=dev)
    xt = (w * scale[:, None]) @ t.T            # p x n row-major = n x p column-major
    xt += noise * torch.randn(p, n, generator=g, device=dev)
    xt -= xt.mean(dim=1, keepdim=True)
    xb = xt.to(torch.bfloat16)
    del xt
    y = (t @ c + 0.1 * torch.randn(n, m, generator=g, device=dev)).T.contiguous()
    bits = xb.view(torch.int16).cpu().numpy().view(np.uint16).T
    yh = y.cpu().numpy().T
    del xb, t, w, y, c
    torch.cuda.empty_cache()
    return bits, yh


def bf16_to_f64(bits, rows=None):
    """FP64 values of BF16 bit patterns (exact), optionally of some rows."""
    b = bits if rows is None else bits[rows]
    out = np.empty(b.shape, dtype=np.float64, order="F")
    step = 4096
    for j0 in range(0, b.shape[1], step):
        blk = np.ascontiguousarray(b[:, j0:j0 + step]).astype(np.uint32) << 16
        out[:, j0:j0 + step] = blk.view(np.float32)
    return out


def plssvd_lda_config(seed=2, n=20_000, p=50_000, k=20, classes=10):
    """The PLS-SVD + LDA configuration: X = T W^T + N(0, 0.1^2) (n x p FP32,
    column-centred) with factor scales 100 * 0.8^i; labels = argmax(T C) + 1
    with C ~ N(0, 1) k x classes. Returns (x, labels), x Fortran-ordered."""
    import torch

    dev = torch.device("cuda")
    g = torch.Generator(device=dev).manual_seed(seed)
    sigma = 100.0 * 0.8 ** torch.arange(k, device=dev, dtype=torch.float32)
    t = torch.randn(n, k, generator=g, device=dev) * sigma
    w = torch.randn(p, k, generator=g, device=dev)
    c = torch.randn(k, classes, generator=g, device=dev)
    xt = w @ t.T
    xt += 0.1 * torch.randn(p, n, generator=g, device=dev)
    xt -= xt.mean(dim=1, keepdim=True)
    lab = (torch.argmax(t @ c, dim=1) + 1).to(torch.int32).cpu().numpy()
    x = xt.cpu().numpy().T
    del xt, t, w, c
    torch.cuda.empty_cache()
    return x, lab
