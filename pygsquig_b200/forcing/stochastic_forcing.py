"""Stochastic forcing (mirrors pygsquig/forcing/stochastic_forcing.py).

The reference draws its noise from jax.random keys.  Here ``key`` is the
random source: a ``torch.Generator`` (its device's generator draws the
noise; a CUDA generator keeps everything on the GPU), a
``numpy.random.Generator`` (drawn on the host, then uploaded: reproducible
against NumPy), an int seed, or None (torch's default generator).  Two
draws the reference takes from split keys are consecutive draws of one
source here.  Noise is built in float64 and returned in the dtype and on
the device of theta_hat; the solvers add it to the stage update in the row
pass (the ``extra`` spectral input).
"""

from __future__ import annotations

import math
from abc import ABC, abstractmethod
from typing import Optional

import numpy as np
import torch

from ..core.grid import fft2
from ..exceptions import ForcingError


def _device(theta_hat, grid):
    return theta_hat.device if isinstance(theta_hat, torch.Tensor) else grid.x.device


def _out(x: torch.Tensor, theta_hat) -> torch.Tensor:
    if isinstance(theta_hat, torch.Tensor) and theta_hat.is_complex():
        return x.to(device=theta_hat.device, dtype=theta_hat.dtype)
    return x


def _normal(key, shape, device) -> torch.Tensor:
    """Standard normal float64 draws of the given shape from ``key``."""
    if isinstance(key, np.random.Generator):
        return torch.as_tensor(key.standard_normal(shape), device=device)
    if isinstance(key, torch.Generator):
        return torch.randn(shape, generator=key, device=key.device, dtype=torch.float64).to(device)
    if isinstance(key, (int, np.integer)):
        g = torch.Generator(device=device).manual_seed(int(key))
        return torch.randn(shape, generator=g, device=device, dtype=torch.float64)
    if key is None:
        return torch.randn(shape, device=device, dtype=torch.float64)
    raise ForcingError(f"unsupported random source {type(key).__name__}")


def _uniform(key, n, device) -> torch.Tensor:
    if isinstance(key, np.random.Generator):
        return torch.as_tensor(key.random(n), device=device)
    if isinstance(key, torch.Generator):
        return torch.rand(n, generator=key, device=key.device, dtype=torch.float64).to(device)
    g = None
    if isinstance(key, (int, np.integer)):
        g = torch.Generator(device=device).manual_seed(int(key))
    return torch.rand(n, generator=g, device=device, dtype=torch.float64)


def _poisson(key, lam: float) -> int:
    if isinstance(key, np.random.Generator):
        return int(key.poisson(lam))
    g = key if isinstance(key, torch.Generator) else None
    if isinstance(key, (int, np.integer)):
        g = torch.Generator().manual_seed(int(key))
    rate = torch.tensor([lam], dtype=torch.float64, device=g.device if g is not None else "cpu")
    return int(torch.poisson(rate, generator=g).item())


def _kmag(grid, device):
    return torch.sqrt(grid.kx**2 + grid.ky**2).to(device)


def _band_mask(grid, device, k_min, k_max):
    k = _kmag(grid, device)
    m = torch.ones_like(k)
    if k_min is not None:
        m = m * (k >= k_min)
    if k_max is not None:
        m = m * (k <= k_max)
    m[0, 0] = 0
    return m


def _real_corners(z: torch.Tensor, N: int) -> torch.Tensor:
    """Imaginary parts of the four self-conjugate modes set to zero
    (stochastic_forcing.py:132-146)."""
    z = z.clone()
    parts = torch.view_as_real(z)
    H = N // 2
    for i, j in ((0, 0), (H, 0), (0, H), (H, H)):
        parts[i, j, 1] = 0
    return z


class StochasticForcing(ABC):
    """stochastic_forcing.py:19-39."""

    @abstractmethod
    def __call__(self, theta_hat, key, dt: float, grid):
        """Forcing increment in spectral space."""


class WhiteNoiseForcing(StochasticForcing):
    """Gaussian noise of std A sqrt(dt) per mode, optional band, four real
    corner modes, rescaled to inject A^2 dt when isotropic, mean zero
    (stochastic_forcing.py:42-162)."""

    def __init__(self, amplitude: float = 0.1, k_min: Optional[float] = None, k_max: Optional[float] = None,
                 isotropy: bool = True):
        if amplitude < 0:
            raise ForcingError("Amplitude must be non-negative")
        self.amplitude, self.k_min, self.k_max, self.isotropy = amplitude, k_min, k_max, isotropy

    def __call__(self, theta_hat, key, dt: float, grid):
        dev, N = _device(theta_hat, grid), grid.N
        std = self.amplitude * math.sqrt(dt)
        re = _normal(key, (N, N), dev) * std
        im = _normal(key, (N, N), dev) * std
        z = torch.complex(re, im)
        if self.k_min is not None or self.k_max is not None:
            z = z * _band_mask(grid, dev, self.k_min, self.k_max)
        z = _real_corners(z, N)
        if self.isotropy:
            e = float(torch.sum(z.abs() ** 2)) / N**4
            if e > 0:
                z = z * math.sqrt(self.amplitude**2 * dt / e)
        z[0, 0] = 0
        return _out(z, theta_hat)


class ColoredNoiseForcing(StochasticForcing):
    """Noise shaped by (k/k_p)^s exp(-((k - k_p)/w)^2), times A sqrt(dt)
    (stochastic_forcing.py:165-241)."""

    def __init__(self, amplitude: float = 0.1, spectral_slope: float = -2.0, k_peak: float = 10.0,
                 k_width: float = 5.0):
        if amplitude < 0:
            raise ForcingError("Amplitude must be non-negative")
        self.amplitude, self.spectral_slope, self.k_peak, self.k_width = amplitude, spectral_slope, k_peak, k_width

    def spectrum(self, grid, device) -> torch.Tensor:
        k = _kmag(grid, device)
        ks = torch.where(k > 0, k, torch.ones_like(k))
        s = (ks / self.k_peak) ** self.spectral_slope * torch.exp(-(((ks - self.k_peak) / self.k_width) ** 2))
        return torch.where(k > 0, s, torch.zeros_like(s))

    def __call__(self, theta_hat, key, dt: float, grid):
        dev, N = _device(theta_hat, grid), grid.N
        z = torch.complex(_normal(key, (N, N), dev), _normal(key, (N, N), dev))
        z = z * torch.sqrt(self.spectrum(grid, dev)) * (self.amplitude * math.sqrt(dt))
        z = _real_corners(z, N)
        z[0, 0] = 0
        return _out(z, theta_hat)


class StochasticVortexForcing(StochasticForcing):
    """Poisson(rate dt) Gaussian vortices s_i exp(-r^2 / (2 R^2)), R =
    size L, at uniform positions, strengths A (1 + std n), random signs
    (stochastic_forcing.py:244-317)."""

    def __init__(self, amplitude: float = 0.1, vortex_size: float = 0.1, injection_rate: float = 1.0,
                 vortex_strength_std: float = 0.2):
        if amplitude < 0:
            raise ForcingError("Amplitude must be non-negative")
        if vortex_size <= 0 or vortex_size > 1:
            raise ForcingError("Vortex size must be in (0, 1]")
        if injection_rate < 0:
            raise ForcingError("Injection rate must be non-negative")
        self.amplitude, self.vortex_size = amplitude, vortex_size
        self.injection_rate, self.vortex_strength_std = injection_rate, vortex_strength_std

    def __call__(self, theta_hat, key, dt: float, grid):
        dev, N = _device(theta_hat, grid), grid.N
        n = _poisson(key, self.injection_rate * dt)
        if n == 0:
            return _out(torch.zeros((N, N), dtype=torch.complex128, device=dev), theta_hat)
        xs = _uniform(key, n, dev) * grid.L
        ys = _uniform(key, n, dev) * grid.L
        strengths = self.amplitude * (1 + self.vortex_strength_std * _normal(key, (n,), dev))
        signs = 2.0 * (_uniform(key, n, dev) < 0.5).double() - 1.0
        x, y = grid.x.to(dev), grid.y.to(dev)
        R2 = (self.vortex_size * grid.L) ** 2
        f = torch.zeros_like(x)
        for i in range(n):  # the reference adds the vortices one by one through ifft2 / fft2
            f = f + strengths[i] * signs[i] * torch.exp(-((x - xs[i]) ** 2 + (y - ys[i]) ** 2) / (2 * R2))
        return _out(fft2(f, grid.L), theta_hat)


class OrnsteinUhlenbeckForcing(StochasticForcing):
    """OU process per mode: z <- e z + A sqrt(2 dt/tau (1 - e^2)) n,
    e = exp(-dt/tau); optional band; four real corners; mean zero
    (stochastic_forcing.py:320-426).  As in the reference, the real and
    imaginary parts of the initial state and of each increment are the same
    draw (one key serves both there)."""

    def __init__(self, amplitude: float = 0.1, correlation_time: float = 1.0, k_min: Optional[float] = None,
                 k_max: Optional[float] = None):
        if amplitude < 0:
            raise ForcingError("Amplitude must be non-negative")
        if correlation_time <= 0:
            raise ForcingError("Correlation time must be positive")
        self.amplitude, self.correlation_time, self.k_min, self.k_max = amplitude, correlation_time, k_min, k_max
        self._ou_state = None

    def __call__(self, theta_hat, key, dt: float, grid):
        dev, N = _device(theta_hat, grid), grid.N
        if self._ou_state is None:
            n0 = _normal(key, (N, N), dev)
            self._ou_state = torch.complex(n0, n0)
        decay = math.exp(-dt / self.correlation_time)
        amp = self.amplitude * math.sqrt(2 * dt / self.correlation_time * (1 - decay**2))
        n = _normal(key, (N, N), dev)
        self._ou_state = decay * self._ou_state + amp * torch.complex(n, n)
        f = self._ou_state
        if self.k_min is not None or self.k_max is not None:
            f = f * _band_mask(grid, dev, self.k_min, self.k_max)
        f = _real_corners(f, N)
        f[0, 0] = 0
        return _out(f, theta_hat)


def create_combined_stochastic_forcing(forcings: list, weights: Optional[list] = None) -> StochasticForcing:
    """Weighted sum with weights normalised to one (stochastic_forcing.py:429-479)."""
    if not forcings:
        raise ForcingError("Must provide at least one forcing")
    if weights is None:
        weights = [1.0] * len(forcings)
    elif len(weights) != len(forcings):
        raise ForcingError("Number of weights must match number of forcings")
    total = sum(weights)
    if total <= 0:
        raise ForcingError("Sum of weights must be positive")
    norm = [w / total for w in weights]

    class CombinedStochasticForcing(StochasticForcing):
        def __init__(self):
            self.forcings, self.weights = forcings, norm

        def __call__(self, theta_hat, key, dt: float, grid):
            out = None
            for f, w in zip(self.forcings, self.weights):
                term = w * f(theta_hat, key, dt, grid)
                out = term if out is None else out + term
            return out

    return CombinedStochasticForcing()
