"""Diagnostics reduced in float64 on the GPU (mirrors
pygsquig/utils/diagnostics.py and scalars/diagnostics.py:156-168)."""

from __future__ import annotations

import numpy as np
import torch

from .._plan import PlanKey, get_plan


def _plan(grid, theta_hat, alpha):
    prec = "float32" if isinstance(theta_hat, torch.Tensor) and theta_hat.dtype == torch.complex64 else "float64"
    return get_plan(PlanKey(N=grid.N, L=float(grid.L), alpha=float(alpha), nu_p=0.0, p=8, precision=prec))


def _diag(theta_hat, grid, alpha):
    pl = _plan(grid, theta_hat, alpha)
    return pl.diagnostics(pl.check_spectrum(theta_hat))


def compute_total_energy(theta_hat, grid, alpha: float) -> float:
    """E = 1/2 sum k2^((alpha-2)/2) |theta_hat|^2 / N^2 (diagnostics.py:171-190)."""
    return float(_diag(theta_hat, grid, alpha)[0])


def compute_enstrophy(theta_hat, grid, alpha: float) -> float:
    """Z = 1/2 sum |k|^(2 alpha) |theta_hat|^2 (diagnostics.py:120-141)."""
    return float(_diag(theta_hat, grid, alpha)[1])


def compute_palinstrophy(theta_hat, grid, alpha: float) -> float:
    """P = 1/2 sum k2^(1+alpha) |theta_hat|^2 / N^2 (diagnostics.py:194-217)."""
    return float(_diag(theta_hat, grid, alpha)[5])


def compute_energy_spectrum(theta_hat, grid, alpha: float):
    """(k_bins, E_k) in min(N/4, 64) linear bins (diagnostics.py:31-84)."""
    pl = _plan(grid, theta_hat, alpha)
    E = pl.energy_spectrum(pl.check_spectrum(theta_hat))
    dk = 2 * np.pi / grid.L
    k_max = grid.N * dk / 2
    n_bins = min(grid.N // 4, 64)
    edges = np.linspace(0, k_max, n_bins + 1)
    return 0.5 * (edges[:-1] + edges[1:]), E


def compute_scalar_variance(scalar_hat, grid) -> float:
    """<(s - <s>)^2> (scalars/diagnostics.py:156-168)."""
    pl = _plan(grid, scalar_hat, 0.0)
    return pl.scalar_variance(pl.check_spectrum(scalar_hat))


def compute_energy_flux(theta_hat, forcing_hat, grid) -> float:
    """Re sum conj(theta_hat) F / N^2 (diagnostics.py:145-167)."""
    if forcing_hat is None:
        return 0.0
    return float((torch.conj(theta_hat) * forcing_hat).real.sum().item()) / grid.N**2
