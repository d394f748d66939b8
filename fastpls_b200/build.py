"""Build the in-tree CUDA library ``fastpls_b200/libfastpls_b200.so`` for sm_100a.

Usage: ``python -m fastpls_b200.build`` (or ``build()`` from Python). The
library is plain C ABI (include/fastpls_b200.h) with no PyTorch dependency.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfastpls_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]


def sources():
    return sorted(glob.glob(os.path.join(SRC, "*.cu")))


def build(verbose: bool = False, jobs: int | None = None) -> str:
    """Compile every .cu to an object (in parallel) and link the shared library."""
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    srcs = sources()
    deps = srcs + glob.glob(os.path.join(SRC, "*.cuh")) + \
        [os.path.join(HERE, os.pardir, "include", "fastpls_b200.h")]
    newest = max(os.path.getmtime(p) for p in deps)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    procs = []
    objs = []
    for src in srcs:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= newest:
            continue
        cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode()))
        elif verbose and out:
            print(out.decode())
    if failed:
        msg = "\n".join(f"--- {s}\n{o}" for s, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
