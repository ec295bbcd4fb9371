"""Damping (mirrors pygsquig/forcing/damping.py:15-131)."""

from __future__ import annotations

import torch

from .._plan import PlanKey, get_plan


def _prec(t):
    return "float32" if isinstance(t, torch.Tensor) and t.dtype == torch.complex64 else "float64"


def _plan(grid, precision, mu, kf, nu_p, p):
    return get_plan(PlanKey(N=grid.N, L=grid.L, alpha=0.0, nu_p=0.0, p=8, precision=precision,
                            damping=(float(mu), float(kf), float(nu_p), int(p))))


def large_scale_damping(theta_hat, grid, mu: float, kf: float) -> torch.Tensor:
    """-mu theta_hat on |k| < kf/2, k = 0 included (damping.py:15-43)."""
    pl = _plan(grid, _prec(theta_hat), mu, kf, 0.0, 8)
    th = pl.check_spectrum(theta_hat)
    if mu == 0:
        return torch.zeros_like(th)
    return pl.damping(th)


def hyperviscosity(theta_hat, grid, nu_p: float, p: int) -> torch.Tensor:
    """-nu_p k2^(p/2) theta_hat, zero at k = 0 (operators.py:185-207)."""
    pl = get_plan(PlanKey(N=grid.N, L=grid.L, alpha=0.0, nu_p=float(nu_p), p=int(p), precision=_prec(theta_hat)))
    return pl.hyperviscosity(pl.check_spectrum(theta_hat))


class CombinedDamping:
    """Large-scale drag plus hyperviscosity (damping.py:49-131)."""

    def __init__(self, mu: float = 0.0, kf: float = 20.0, nu_p: float = 0.0, p: int = 8):
        self.mu = mu
        self.kf = kf
        self.nu_p = nu_p
        self.p = p
        if p not in [2, 4, 8]:
            raise ValueError(f"p must be 2, 4, or 8, got {p}")

    def plan_tuple(self):
        return (float(self.mu), float(self.kf), float(self.nu_p), int(self.p))

    def __call__(self, theta_hat, grid=None, **kwargs) -> torch.Tensor:
        if grid is None:
            raise TypeError("CombinedDamping needs the grid (call damping(theta_hat, grid))")
        pl = _plan(grid, _prec(theta_hat), *self.plan_tuple())
        return pl.damping(pl.check_spectrum(theta_hat))

    def get_diagnostics(self, theta_hat, grid) -> dict:
        pl = _plan(grid, _prec(theta_hat), *self.plan_tuple())
        th = pl.check_spectrum(theta_hat)
        ls = _plan(grid, _prec(theta_hat), self.mu, self.kf, 0.0, self.p).damping(th)
        ss = hyperviscosity(th, grid, self.nu_p, self.p)
        lsd = -pl.inner(th, ls)
        ssd = -pl.inner(th, ss)
        k = grid.k1d
        import numpy as np
        kk = np.sqrt(k[:, None] ** 2 + k[None, :] ** 2)
        return {
            "large_scale_dissipation": lsd,
            "small_scale_dissipation": ssd,
            "total_dissipation": lsd + ssd,
            "n_large_scale_modes": int(np.sum(kk < self.kf / 2)),
            "mu": self.mu,
            "nu_p": self.nu_p,
        }
