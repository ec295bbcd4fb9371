"""Build libsqg.so in-tree with nvcc for sm_100a.

    python -m pygsquig_b200.build [--force]

Each translation unit is compiled to an object under ``_build/`` (rebuilt
when it or a header it includes changed) and the objects are linked into
``libsqg.so`` beside this file.  The library counts as up to date when it is
newer than every source and header, so a copy that carries the library but
not the objects does not rebuild.
"""

from __future__ import annotations

import fcntl
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
_INST = [f"sqg_inst_{t}_{r}.cu" for t in ("f32", "f64") for r in "abc"] + ["sqg_inst_multi.cu"]
SRCS = [os.path.join(CSRC, f) for f in ["sqg_capi.cu"] + _INST + ["closure_conv.cu", "closure_ops.cu"]]
# headers each unit includes (a change rebuilds the unit)
_PASS_HDRS = ["pdl.cuh", "sqg_fft.cuh", "sqg_tma.cuh", "sqg_kernels.cuh", "sqg_launch.cuh"]
DEPS = {
    "sqg_capi.cu": _PASS_HDRS + ["sqg_aux.cuh", "../../include/sqg.h"],
    "closure_conv.cu": ["pdl.cuh", "closure_act.cuh", "../../include/sqg_closure.h"],
    "closure_ops.cu": ["pdl.cuh", "closure_act.cuh", "../../include/sqg_closure.h"],
}
DEPS.update({f: _PASS_HDRS for f in _INST})
OUT = os.path.join(HERE, "libsqg.so")
OBJ_DIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17"] + ARCH + ["-lineinfo", "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _obj(src: str) -> str:
    return os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + ".o")


def _deps(src: str):
    return [src] + [os.path.normpath(os.path.join(CSRC, d)) for d in DEPS[os.path.basename(src)]]


def _stale(target: str, inputs) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in inputs)


def up_to_date() -> bool:
    """The library exists and is newer than every source and header."""
    return not _stale(OUT, [p for s in SRCS for p in _deps(s)])


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(OBJ_DIR, exist_ok=True)
    with open(os.path.join(OBJ_DIR, ".lock"), "w") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)  # one build at a time (tests and scripts may race)
        if not force and up_to_date():
            return OUT
        return _build(force, verbose)


def _build(force: bool, verbose: bool) -> str:
    t_start = time.time()
    os.makedirs(OBJ_DIR, exist_ok=True)
    objs, jobs = [], []
    for s in SRCS:
        o = _obj(s)
        if force or _stale(o, _deps(s)):
            cmd = [nvcc()] + NVCC_FLAGS + ["-c", "-o", o + ".tmp", s]
            if verbose:
                print(" ".join(cmd))
            jobs.append((o, subprocess.Popen(cmd)))
        objs.append(o)
    failed = [o for o, pr in jobs if pr.wait() != 0]  # the units compile in parallel
    if failed:
        raise subprocess.CalledProcessError(1, "nvcc", output=f"failed: {failed}")
    for o, _ in jobs:
        os.replace(o + ".tmp", o)
    cmd = [nvcc()] + ARCH + ["-shared", "-o", OUT + ".tmp"] + objs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    os.utime(OUT, (t_start, t_start))  # a source edited during the build makes the library stale
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
