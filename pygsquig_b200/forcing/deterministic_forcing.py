"""Deterministic forcing patterns (mirrors pygsquig/forcing/deterministic_forcing.py).

Each pattern is a physical field built on the device from the grid's float64
coordinates, transformed once by the library's forward transform and kept;
a call returns the kept spectrum times the current amplitude in the dtype
and on the device of theta_hat.  The solvers add such a term to the stage
update inside the row pass (the ``extra`` spectral input), so a forcing
costs one device multiply per stage.  Calls follow the reference's
interface ``forcing(theta_hat, key, dt, grid)``; use them in a solver step
as ``forcing=lambda th, **kw: f(th, None, dt, grid)``.
"""

from __future__ import annotations

import math
from abc import ABC, abstractmethod
from typing import Optional

import torch

from ..core.grid import fft2, ifft2
from ..exceptions import ForcingError


def _positive(value, name):
    if not isinstance(value, (float, int)) or isinstance(value, bool) or value <= 0:
        raise ForcingError(f"{name} must be positive number, got {value}")
    return float(value)


def _positive_int(value, name):
    if not isinstance(value, int) or isinstance(value, bool) or value < 1:
        raise ForcingError(f"{name} must be positive integer, got {value}")
    return value


def _direction(value):
    if value not in ("x", "y"):
        raise ForcingError(f"direction must be 'x' or 'y', got {value}")
    return value


class DeterministicForcing(ABC):
    """deterministic_forcing.py:20-71."""

    @abstractmethod
    def __call__(self, theta_hat, key, dt: float, grid):
        """Forcing spectrum F_hat for one call."""

    def get_diagnostics(self, theta_hat, forcing, grid) -> dict:
        """<theta F> and sum |F_hat|^2 / N^2 (deterministic_forcing.py:48-71)."""
        theta = ifft2(theta_hat)
        force = ifft2(forcing)
        return {
            "injection_rate": float(torch.mean(theta.double() * force.double())),
            "forcing_power": float(torch.sum(forcing.abs().double() ** 2)) / grid.N**2,
            "forcing_type": self.__class__.__name__,
        }


class _StaticPattern(DeterministicForcing):
    """A fixed physical pattern times a (possibly time-dependent) amplitude."""

    def _pattern(self, grid) -> torch.Tensor:
        raise NotImplementedError

    def _spectrum(self, grid, like: torch.Tensor) -> torch.Tensor:
        cache = self.__dict__.setdefault("_cache", {})
        key = (id(grid), grid.N, float(grid.L), like.dtype, str(like.device))
        if key not in cache:
            cache.clear()
            f_hat = fft2(self._pattern(grid).to(torch.float64), grid.L)
            cache[key] = f_hat.to(device=like.device, dtype=like.dtype)
        return cache[key]

    def _like(self, theta_hat, grid):
        if isinstance(theta_hat, torch.Tensor) and theta_hat.is_complex():
            return theta_hat
        return torch.empty((grid.N, grid.N), dtype=torch.complex128, device=grid.x.device)

    def _amplitude(self, dt) -> float:
        return 1.0

    def __call__(self, theta_hat, key, dt: float, grid):
        like = self._like(theta_hat, grid)
        return self._spectrum(grid, like) * self._amplitude(dt)


class TaylorGreenForcing(_StaticPattern):
    """F = A sin(k x) cos(k y), A cos(t) when time_dependent, t advanced by
    dt on every call (deterministic_forcing.py:74-122)."""

    def __init__(self, amplitude: float = 1.0, k: int = 2, time_dependent: bool = False):
        self.amplitude = _positive(amplitude, "amplitude")
        self.k = _positive_int(k, "k")
        self.time_dependent = time_dependent

    def _pattern(self, grid):
        kk = self.k * 2 * math.pi / grid.L
        return torch.sin(kk * grid.x) * torch.cos(kk * grid.y)

    def _amplitude(self, dt):
        t = float(getattr(self, "_time", 0.0))
        self._time = t + dt
        return self.amplitude * math.cos(t) if self.time_dependent else self.amplitude


class KolmogorovForcing(_StaticPattern):
    """F = A sin(k y) (or sin(k x)) (deterministic_forcing.py:125-169)."""

    def __init__(self, amplitude: float = 1.0, k: int = 4, direction: str = "y"):
        self.amplitude = _positive(amplitude, "amplitude")
        self.k = _positive_int(k, "k")
        self.direction = _direction(direction)

    def _pattern(self, grid):
        kk = self.k * 2 * math.pi / grid.L
        return torch.sin(kk * (grid.y if self.direction == "y" else grid.x))

    def _amplitude(self, dt):
        return self.amplitude


class CheckerboardForcing(_StaticPattern):
    """F = A sign(sin(kx x) sin(ky y)) (deterministic_forcing.py:172-213)."""

    def __init__(self, amplitude: float = 1.0, kx: int = 4, ky: Optional[int] = None):
        self.amplitude = _positive(amplitude, "amplitude")
        self.kx = _positive_int(kx, "kx")
        self.ky = _positive_int(ky if ky is not None else kx, "ky")

    def _pattern(self, grid):
        kx = self.kx * 2 * math.pi / grid.L
        ky = self.ky * 2 * math.pi / grid.L
        return torch.sign(torch.sin(kx * grid.x) * torch.sin(ky * grid.y))

    def _amplitude(self, dt):
        return self.amplitude


class ShearLayerForcing(_StaticPattern):
    """Linear A (y/L - 1/2) or A tanh((y - y0)/width) profile
    (deterministic_forcing.py:216-278)."""

    def __init__(self, amplitude: float = 1.0, profile: str = "linear", direction: str = "y",
                 center: Optional[float] = None, width: float = 0.1):
        self.amplitude = _positive(amplitude, "amplitude")
        if profile not in ("linear", "tanh"):
            raise ForcingError(f"profile must be 'linear' or 'tanh', got {profile}")
        self.profile = profile
        self.direction = _direction(direction)
        self.center = center
        self.width = _positive(width, "width")

    def _pattern(self, grid):
        c = grid.y if self.direction == "y" else grid.x
        if self.profile == "linear":
            return c / grid.L - 0.5
        center = self.center if self.center is not None else grid.L / 2
        return torch.tanh((c - center) / self.width)

    def _amplitude(self, dt):
        return self.amplitude


class VortexPairForcing(_StaticPattern):
    """Sum of Gaussian vortices Gamma / (pi r^2) exp(-d^2 / r^2) with periodic
    distances (deterministic_forcing.py:281-344)."""

    def __init__(self, vortices: list, amplitude_scale: float = 1.0):
        self.vortices = []
        for v in vortices:
            if len(v) != 4:
                raise ForcingError("Each vortex must be (x, y, circulation, radius)")
            x, y, circ, radius = v
            if not isinstance(radius, (float, int)) or radius <= 0:
                raise ForcingError(f"vortex radius must be positive, got {radius}")
            self.vortices.append({"x": float(x), "y": float(y), "circulation": float(circ), "radius": float(radius)})
        self.amplitude_scale = _positive(amplitude_scale, "amplitude_scale")

    @staticmethod
    def _periodic_distance(coord, center: float, L: float):
        d = coord - center
        d = torch.where(d > L / 2, d - L, d)
        return torch.where(d < -L / 2, d + L, d)

    def _pattern(self, grid):
        f = torch.zeros_like(grid.x)
        for v in self.vortices:
            dx = self._periodic_distance(grid.x, v["x"], grid.L)
            dy = self._periodic_distance(grid.y, v["y"], grid.L)
            f = f + v["circulation"] / (math.pi * v["radius"] ** 2) * torch.exp(-(dx**2 + dy**2) / v["radius"] ** 2)
        return f

    def _amplitude(self, dt):
        return self.amplitude_scale


class TimeModulatedForcing(DeterministicForcing):
    """Base pattern times sin / cos(2 pi f t + phase), exp(-r t) or
    min(r t, 1); t advanced by dt on every call
    (deterministic_forcing.py:347-420)."""

    def __init__(self, base_forcing: DeterministicForcing, modulation: str = "sine", frequency: float = 1.0,
                 decay_rate: float = 1.0, phase: float = 0.0):
        if not isinstance(base_forcing, DeterministicForcing):
            raise ForcingError("base_forcing must be a DeterministicForcing instance")
        if modulation not in ("sine", "cosine", "exponential", "ramp"):
            raise ForcingError(f"Unknown modulation type: {modulation}")
        self.base_forcing = base_forcing
        self.modulation = modulation
        self.frequency = _positive(frequency, "frequency")
        self.decay_rate = _positive(decay_rate, "decay_rate")
        self.phase = phase
        self._time = 0.0

    def _factor(self, t: float) -> float:
        if self.modulation == "sine":
            return math.sin(2 * math.pi * self.frequency * t + self.phase)
        if self.modulation == "cosine":
            return math.cos(2 * math.pi * self.frequency * t + self.phase)
        if self.modulation == "exponential":
            return math.exp(-self.decay_rate * t)
        return min(t * self.decay_rate, 1.0)

    def __call__(self, theta_hat, key, dt: float, grid):
        base = self.base_forcing(theta_hat, key, dt, grid)
        t = self._time
        self._time = t + dt
        return base * self._factor(t)

    def get_diagnostics(self, theta_hat, forcing, grid) -> dict:
        d = self.base_forcing.get_diagnostics(theta_hat, forcing, grid)
        d["modulation_type"] = self.modulation
        d["current_time"] = self._time
        return d


class CombinedDeterministicForcing(DeterministicForcing):
    """Weighted sum of patterns (deterministic_forcing.py:423-464)."""

    def __init__(self, forcings: list):
        self.forcings = []
        for weight, forcing in forcings:
            if not isinstance(forcing, DeterministicForcing):
                raise ForcingError(f"Each forcing must be DeterministicForcing, got {type(forcing)}")
            self.forcings.append((float(weight), forcing))

    def __call__(self, theta_hat, key, dt: float, grid):
        total = None
        for w, f in self.forcings:
            term = w * f(theta_hat, key, dt, grid)
            total = term if total is None else total + term
        if total is None:
            like = theta_hat if isinstance(theta_hat, torch.Tensor) else torch.as_tensor(theta_hat)
            return torch.zeros_like(like)
        return total

    def get_diagnostics(self, theta_hat, forcing, grid) -> dict:
        d = super().get_diagnostics(theta_hat, forcing, grid)
        d["n_components"] = len(self.forcings)
        return d


def make_taylor_green_forcing(amplitude: float = 1.0, k: int = 2, time_decay: bool = False) -> DeterministicForcing:
    return TaylorGreenForcing(amplitude=amplitude, k=k, time_dependent=time_decay)


def make_kolmogorov_forcing(amplitude: float = 1.0, k: int = 4, direction: str = "y") -> DeterministicForcing:
    return KolmogorovForcing(amplitude=amplitude, k=k, direction=direction)


def make_oscillating_forcing(base_pattern: str = "taylor_green", frequency: float = 1.0,
                             **kwargs) -> DeterministicForcing:
    """deterministic_forcing.py:499-524."""
    bases = {"taylor_green": TaylorGreenForcing, "kolmogorov": KolmogorovForcing,
             "checkerboard": CheckerboardForcing}
    if base_pattern not in bases:
        raise ForcingError(f"Unknown base pattern: {base_pattern}")
    return TimeModulatedForcing(base_forcing=bases[base_pattern](**kwargs), modulation="sine", frequency=frequency)
