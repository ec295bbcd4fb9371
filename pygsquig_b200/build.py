"""Build libsqg.so in-tree with nvcc for sm_100a.

    python -m pygsquig_b200.build [--force]
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRCS = [os.path.join(HERE, "csrc", f) for f in ("sqg_capi.cu", "closure_conv.cu", "closure_ops.cu")]
DEPS = [os.path.join(HERE, "csrc", f) for f in ("sqg_fft.cuh", "sqg_kernels.cuh", "sqg_aux.cuh")] + [
    os.path.join(ROOT, "include", f) for f in ("sqg.h", "sqg_closure.h")]
OUT = os.path.join(HERE, "libsqg.so")

NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-shared"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(p) <= t for p in SRCS + DEPS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", OUT + ".tmp"] + SRCS
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
