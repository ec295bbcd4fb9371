"""Ring forcing (mirrors pygsquig/forcing/ring_forcing.py:16-237).

The random phases are drawn on the host (e.g. ``numpy.random.default_rng``)
and passed in through the ``key`` argument -- the reference's injection point
``_generate_random_phases`` (ring_forcing.py:78-92).  ``key`` is either a 1-D
array of phases for the ring modes in row-major order of the ring mask, or a
full (N, N) array of phases.
"""

from __future__ import annotations

import math
from typing import Optional

import numpy as np
import torch

from .._plan import PlanKey, get_plan


def _prec(t):
    return "float32" if isinstance(t, torch.Tensor) and t.dtype == torch.complex64 else "float64"


class RingForcing:
    """Ring forcing with energy injection rescaled to <theta F> = epsilon."""

    def __init__(self, kf: float, dk: float = 1.0, epsilon: float = 0.1, tau_f: float = 0.0,
                 amplitude: Optional[float] = None):
        self.kf = kf
        self.dk = dk
        self.epsilon = epsilon
        self.tau_f = tau_f
        self.amplitude = math.sqrt(epsilon) if amplitude is None else amplitude
        self.forcing_state = None

    # plan parameters carried by a solver plan
    def plan_tuple(self):
        return (float(self.kf), float(self.dk), float(self.epsilon), float(self.tau_f), float(self.amplitude))

    def _plan(self, grid, precision="float64"):
        return get_plan(PlanKey(N=grid.N, L=grid.L, alpha=0.0, nu_p=0.0, p=8, precision=precision,
                                ring=self.plan_tuple()))

    def _get_forcing_mask(self, grid) -> torch.Tensor:
        """|sqrt(k2) - kf| <= dk/2 (ring_forcing.py:64-76)."""
        return torch.abs(torch.sqrt(grid.k2) - self.kf) <= self.dk / 2

    def n_modes(self, grid) -> int:
        k = grid.k1d
        k2 = k[:, None] ** 2 + k[None, :] ** 2
        return int(np.sum(np.abs(np.sqrt(k2) - self.kf) <= self.dk / 2))

    def draw_phases(self, rng: np.random.Generator, grid, n_steps: Optional[int] = None) -> np.ndarray:
        """Uniform phases in [0, 2 pi) for the ring modes (one row per step)."""
        n = self.n_modes(grid)
        shape = (n,) if n_steps is None else (n_steps, n)
        return rng.uniform(0.0, 2 * np.pi, size=shape)

    def _generate_random_phases(self, key, shape):
        """Unit-amplitude phase factors exp(i phi) of a host phase array."""
        ph = torch.as_tensor(np.asarray(key, dtype=np.float64))
        return torch.polar(torch.ones_like(ph), ph)

    def bind(self, key, dt: float, grid) -> "BoundRingForcing":
        """The forcing callable the reference driver builds (run.py:382-383)."""
        return BoundRingForcing(self, key, dt, grid)

    def __call__(self, theta_hat, key, dt: float, grid) -> torch.Tensor:
        """Forcing spectrum for one call (ring_forcing.py:119-170)."""
        pl = self._plan(grid, _prec(theta_hat))
        th = pl.check_spectrum(theta_hat)
        return pl.ring_forcing(th, pl.phases_tensor(key), dt)

    def get_diagnostics(self, theta_hat, forcing, grid) -> dict:
        """ring_forcing.py:172-201."""
        pl = self._plan(grid, _prec(theta_hat))
        th = pl.check_spectrum(theta_hat)
        f = pl.check_spectrum(forcing, "forcing")
        mask = self._get_forcing_mask(grid)
        return {
            "injection_rate": pl.inner(th, f),
            "forcing_power": float((torch.abs(f) ** 2 * mask).sum().item()),
            "n_forced_modes": int(mask.sum().item()),
            "target_epsilon": self.epsilon,
        }


class BoundRingForcing:
    """forcing(theta_hat, **kw) -> RingForcing(theta_hat, key, dt, grid).

    A solver recognises this object and runs the forcing inside its fused
    stage kernels instead of calling it.
    """

    def __init__(self, ring: RingForcing, key, dt, grid):
        self.ring, self.key, self.dt, self.grid = ring, key, dt, grid

    def __call__(self, theta_hat, **kwargs):
        return self.ring(theta_hat, self.key, self.dt, self.grid)
