"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, validates plans like the reference validates solvers, and
builds grid masks bit-identical to the reference's float64 expressions."""

import ctypes as C
import os
import re

import numpy as np
import pytest

from pygsquig_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = "".join(open(os.path.join(ROOT, "include", f)).read() for f in sorted(os.listdir(os.path.join(ROOT, "include")))
                  if f.endswith(".h"))
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(sqg_\w+)\s*\(", src, flags=re.M)))


def test_exports_every_header_symbol(lib):
    syms = header_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(lib, s), s
        assert s in _lib.SIGNATURES, f"{s} missing from the ctypes table"
    assert lib.sqg_version() >= 1


def make_desc(N=32, L=2 * np.pi, alpha=1.0, p=8, **kw):
    d = _lib.SqgDesc()
    d.N, d.L, d.alpha, d.p = N, L, alpha, p
    d.p_damp = 8
    for k, v in kw.items():
        setattr(d, k, v)
    return d


def create(lib, d):
    h = C.c_void_p()
    rc = lib.sqg_plan_create(C.byref(d), C.byref(h))
    return rc, h


@pytest.mark.parametrize("kw,msg", [
    (dict(N=31), "N must be even"),
    (dict(N=48), "power of two"),
    (dict(alpha=3.0), "alpha must be in"),
    (dict(alpha=-3.0), "alpha must be in"),
    (dict(p=3), "p must be 2, 4, or 8"),
    (dict(has_damping=1, p_damp=5), "p must be 2, 4, or 8"),
])
def test_plan_validation(lib, kw, msg):
    rc, h = create(lib, make_desc(**kw))
    assert rc == _lib.SQG_ERR_INVALID
    with pytest.raises(ValueError, match=msg):
        _lib.check(rc)


def test_workspace_required(lib):
    rc, h = create(lib, make_desc())
    assert rc == 0
    x = C.c_void_p(0)
    rc = lib.sqg_rhs(h, x, x, None)
    assert rc == _lib.SQG_ERR_WORKSPACE
    assert b"workspace" in lib.sqg_last_error_string()
    lib.sqg_plan_destroy(h)


def ref_grid(N, L):
    dx = L / N
    k = np.fft.fftfreq(N, d=dx) * 2 * np.pi
    kx, ky = np.meshgrid(k, k, indexing="ij")
    return k, kx**2 + ky**2


@pytest.mark.parametrize("N,L", [(16, 2 * np.pi), (32, 1.0), (256, 2 * np.pi), (1024, 2 * np.pi), (4096, 2 * np.pi),
                                 (128, 3.7)])
def test_masks_bitexact(lib, N, L):
    kfd = 20.0
    rc, h = create(lib, make_desc(N=N, L=L, has_damping=1, mu=0.1, kf_damp=kfd, p_damp=8))
    assert rc == 0
    k = (C.c_double * N)()
    dm = (C.c_int32 * N)()
    dr = (C.c_int32 * N)()
    assert lib.sqg_plan_host_tables(h, k, dm, dr) == 0
    kref, k2 = ref_grid(N, L)
    assert np.array_equal(np.array(k[:]), kref)
    my = np.minimum(np.arange(N), N - np.arange(N))
    dealias = np.array(dm[:])[:, None] >= my[None, :]
    assert np.array_equal(dealias, np.sqrt(k2) < (2.0 / 3.0) * (np.pi * N / L))
    drag = np.array(dr[:])[:, None] >= my[None, :]
    assert np.array_equal(drag, np.sqrt(k2) < kfd / 2)
    lib.sqg_plan_destroy(h)


@pytest.mark.parametrize("N,kf,dk,count", [(64, 10.0, 2.0, None), (1024, 40.0, 2.0, 496), (128, 20.0, 1.0, None),
                                           (4096, 100.0, 2.0, None), (32, 0.5, 3.0, None), (16, 8.0, 1.0, None)])
def test_ring_modes_order(lib, N, kf, dk, count):
    rc, h = create(lib, make_desc(N=N, has_ring=1, ring_kf=kf, ring_dk=dk, ring_epsilon=0.1, ring_amplitude=0.3))
    assert rc == 0
    n = C.c_int32()
    lib.sqg_ring_mode_count(h, C.byref(n))
    _, k2 = ref_grid(N, 2 * np.pi)
    mask = np.abs(np.sqrt(k2) - kf) <= dk / 2
    assert n.value == mask.sum()
    if count is not None:
        assert n.value == count
    ix = (C.c_int32 * max(n.value, 1))()
    iy = (C.c_int32 * max(n.value, 1))()
    lib.sqg_ring_modes(h, ix, iy)
    rix, riy = np.nonzero(mask)  # row-major order
    assert np.array_equal(np.array(ix[: n.value]), rix)
    assert np.array_equal(np.array(iy[: n.value]), riy)
    lib.sqg_plan_destroy(h)


def test_workspace_size_scales(lib):
    sizes = {}
    for prec in (0, 1):
        rc, h = create(lib, make_desc(N=1024, precision=prec))
        b = C.c_size_t()
        lib.sqg_plan_workspace_bytes(h, C.byref(b))
        sizes[prec] = b.value
        lib.sqg_plan_destroy(h)
    # acc + stage + 4 half + 1 half transformed buffers dominate
    assert sizes[0] > 1.9 * sizes[1] > 0
    assert sizes[0] < 200 * 1024 * 1024
