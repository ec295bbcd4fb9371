"""The no-allocation RHS entry point, checked against the plan-based one.

``sqg_rhs_noalloc`` serves callers that cannot allocate device memory (a host
application that reserves all device memory through its own allocator, or a
loop in which cudaMalloc/cudaFree are banned because they can synchronise the
device): it takes a descriptor and the caller's input/output spectra and keeps
its tables and intermediate fields in a static device array (N <= 256).
This test calls it through the C ABI twice in a row, with different grids,
precisions and inputs, and compares each result with ``sqg_rhs`` (plan plus
caller-provided workspace) at the tolerances the other parity tests use.
It lives in its own file so that pytest collects it last.
"""

import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TWO_PI = 2 * np.pi


def _desc(_lib, N, prec, alpha, nu, p, L=TWO_PI):
    d = _lib.SqgDesc()
    d.N, d.L, d.alpha, d.nu_p, d.p = N, L, alpha, nu, p
    d.precision = _lib.SQG_F64 if prec == "float64" else _lib.SQG_F32
    d.p_damp = 8
    return d


def _field(N, seed):
    rng = np.random.default_rng(seed)
    x = np.arange(N) * TWO_PI / N
    X, Y = np.meshgrid(x, x, indexing="ij")
    f = np.zeros((N, N))
    for _ in range(8):
        kx, ky = rng.integers(-7, 8, size=2)
        f += rng.standard_normal() * np.cos(kx * X + ky * Y + rng.uniform(0, TWO_PI))
    return np.fft.fft2(f)


def test_rhs_noalloc_matches_plan_rhs_twice():
    from pygsquig_b200 import _lib
    from pygsquig_b200._plan import PlanKey, get_plan
    from pygsquig_b200.build import build

    build()
    lib = _lib.load()
    assert torch.cuda.is_available()
    cases = [  # two calls in a row, different grid / precision / physics
        (256, "float64", 1.0, 1e-6, 8, 11, 1e-12),
        (64, "float32", 0.5, 1e-3, 4, 12, 2e-5),
    ]
    for N, prec, alpha, nu, p, seed, tol in cases:
        cdt = torch.complex128 if prec == "float64" else torch.complex64
        th = torch.as_tensor(_field(N, seed)).to("cuda", cdt).contiguous()
        out = torch.empty_like(th)
        stream = torch.cuda.current_stream().cuda_stream
        d = _desc(_lib, N, prec, alpha, nu, p)
        _lib.check(lib.sqg_rhs_noalloc(C.byref(d), th.data_ptr(), out.data_ptr(), stream))
        ref = get_plan(PlanKey(N=N, L=TWO_PI, alpha=alpha, nu_p=nu, p=p, precision=prec)).rhs(th)
        torch.cuda.synchronize()
        a = out.cpu().numpy().astype(np.complex128)
        b = ref.cpu().numpy().astype(np.complex128)
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert err < tol, (N, prec, err)


def test_rhs_noalloc_rejects_oversize_grid():
    from pygsquig_b200 import _lib
    from pygsquig_b200.build import build

    build()
    lib = _lib.load()
    d = _desc(_lib, 512, "float64", 1.0, 0.0, 8)
    x = C.c_void_p(0)
    rc = lib.sqg_rhs_noalloc(C.byref(d), 1, 1, x)
    assert rc == _lib.SQG_ERR_INVALID
    with pytest.raises(ValueError, match="N must be a power of two in \\[8, 256\\]"):
        _lib.check(rc)
