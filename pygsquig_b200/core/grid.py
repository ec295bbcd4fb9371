"""Grid and transforms (mirrors pygsquig/core/grid.py).

``make_grid`` builds the coordinate and wavenumber arrays with the reference's
float64 expressions (grid.py:84-105) on the host, so they are bit-identical,
and keeps them as torch tensors on the current CUDA device (CPU when no GPU
is present, for host-side use only).  ``fft2``/``ifft2`` run the library's
own transform passes; there is no library-FFT or CPU fallback.
"""

from __future__ import annotations

import numpy as np
import torch

from .._plan import PlanKey, get_plan


def _device():
    return torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else torch.device("cpu")


class Grid:
    """Grid of a doubly periodic [0, L)^2 domain with N x N points.

    Attributes mirror the reference (grid.py:15-51): N, L, x, y, kx, ky, k2,
    dealias_mask (torch tensors, float64 / bool, shape (N, N)).
    """

    def __init__(self, N, L, x, y, kx, ky, k2, dealias_mask, k1d):
        self.N = N
        self.L = L
        self.x = x
        self.y = y
        self.kx = kx
        self.ky = ky
        self.k2 = k2
        self.dealias_mask = dealias_mask
        self.k1d = k1d  # numpy float64 fftfreq(N, L/N) * 2 pi

    def __repr__(self):
        return f"Grid(N={self.N}, L={self.L})"


def make_grid(N: int, L: float) -> Grid:
    """Create a Grid (grid.py:72-107).  N must be even; the GPU kernels need a
    power of two in [8, 4096]."""
    if N % 2 != 0:
        raise ValueError(f"N must be even, got {N}")
    dx = L / N
    x1d = np.arange(N) * dx
    x, y = np.meshgrid(x1d, x1d, indexing="ij")
    k1d = np.fft.fftfreq(N, d=dx) * 2 * np.pi
    kx, ky = np.meshgrid(k1d, k1d, indexing="ij")
    k2 = kx**2 + ky**2
    k_max = np.pi * N / L
    dealias_mask = np.sqrt(k2) < (2.0 / 3.0) * k_max
    dev = _device()
    t = lambda a: torch.as_tensor(a, device=dev)  # noqa: E731
    return Grid(N, L, t(x), t(y), t(kx), t(ky), t(k2), t(dealias_mask), k1d)


def _transform_plan(N: int, L: float, precision: str):
    return get_plan(PlanKey(N=N, L=L, alpha=0.0, nu_p=0.0, p=8, precision=precision))


def _precision_of(t) -> str:
    if isinstance(t, torch.Tensor):
        return "float32" if t.dtype in (torch.float32, torch.complex64) else "float64"
    return "float64"


def fft2(field, L: float = 2 * np.pi) -> torch.Tensor:
    """Unnormalised forward 2-D FFT of a real field (grid.py:110-124)."""
    prec = _precision_of(field)
    N = field.shape[0]
    pl = _transform_plan(N, L, prec)
    return pl.to_spectral(pl.check_real(field))


def ifft2(field_hat, L: float = 2 * np.pi) -> torch.Tensor:
    """Inverse 2-D FFT with 1/N^2, real part (grid.py:127-138)."""
    prec = _precision_of(field_hat)
    N = field_hat.shape[0]
    pl = _transform_plan(N, L, prec)
    return pl.to_physical(pl.check_spectrum(field_hat))
