"""CFL-based adaptive time stepping (mirrors pygsquig/core/adaptive_timestep.py).

The velocity comes from the library's transform passes and its maximum
speed from a device reduction (sqg_max_speed); the step-size rules are the
reference's, evaluated on the host from that one number per step.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any, Optional

import numpy as np
import torch

from .._plan import PlanKey, get_plan


@dataclass
class CFLConfig:
    """adaptive_timestep.py:18-56 (same fields, defaults and validation)."""

    cfl_safety: float = 0.8
    dt_min: float = 1e-8
    dt_max: float = 1.0
    growth_factor: float = 1.1
    shrink_factor: float = 0.5
    target_cfl: float = 0.5
    advection_weight: float = 1.0

    def __post_init__(self):
        if not 0 < self.cfl_safety <= 1:
            raise ValueError(f"cfl_safety must be in (0, 1], got {self.cfl_safety}")
        if not 0 < self.target_cfl <= 1:
            raise ValueError(f"target_cfl must be in (0, 1], got {self.target_cfl}")
        if self.dt_min >= self.dt_max:
            raise ValueError(f"dt_min ({self.dt_min}) must be less than dt_max ({self.dt_max})")
        if self.growth_factor <= 1:
            raise ValueError(f"growth_factor must be > 1, got {self.growth_factor}")
        if not 0 < self.shrink_factor < 1:
            raise ValueError(f"shrink_factor must be in (0, 1), got {self.shrink_factor}")


def _field_plan(t):
    """Transform/diagnostic plan for an (N, N) field: float32/complex64 data
    use the FP32 plan, everything else the FP64 one."""
    if isinstance(t, torch.Tensor):
        single = t.dtype in (torch.float32, torch.complex64)
    else:
        single = np.asarray(t).dtype in (np.dtype(np.float32), np.dtype(np.complex64))
    prec = "float32" if single else "float64"
    return get_plan(PlanKey(N=int(t.shape[0]), L=2 * math.pi, alpha=0.0, nu_p=0.0, p=8, precision=prec, role="aux"))


def compute_max_velocity(u: torch.Tensor, v: torch.Tensor) -> float:
    """max sqrt(u^2 + v^2) over the grid (adaptive_timestep.py:59-72)."""
    pl = _field_plan(u)
    return pl.max_speed(pl.check_real(u, "u"), pl.check_real(v, "v"))


def compute_advection_cfl(u: torch.Tensor, v: torch.Tensor, dx: float) -> float:
    """Largest step with advective CFL number 1 (adaptive_timestep.py:75-92)."""
    return dx / max(compute_max_velocity(u, v), 1e-10)


def compute_diffusion_cfl(grid, nu: float, p: int = 2) -> float:
    """Largest step of the (hyper)diffusion condition (adaptive_timestep.py:95-129)."""
    if nu == 0:
        return math.inf
    dx = grid.L / grid.N
    k_max = math.pi * grid.N / grid.L
    if p == 1:
        return 0.25 * dx**2 / nu
    return dx ** (2 * p) / (nu * k_max ** (2 * p - 2))


def compute_timestep(u, v, grid, config: CFLConfig, nu_p: float = 0.0, p: int = 8,
                     current_dt: Optional[float] = None) -> tuple[float, dict[str, Any]]:
    """New step and diagnostics (adaptive_timestep.py:132-199)."""
    return timestep_from_speed(compute_max_velocity(u, v), grid, config, nu_p, p, current_dt)


def timestep_from_speed(vmax: float, grid, config: CFLConfig, nu_p: float = 0.0, p: int = 8,
                        current_dt: Optional[float] = None) -> tuple[float, dict[str, Any]]:
    """The step-size rule of compute_timestep given the maximum speed."""
    dx = grid.L / grid.N
    dt_adv = dx / max(vmax, 1e-10)
    dt_diff = compute_diffusion_cfl(grid, nu_p, p)
    dt_safe = config.cfl_safety * min(dt_adv, dt_diff)
    if current_dt is not None:
        dt_safe = min(dt_safe, current_dt * config.growth_factor)
        if current_dt / dt_adv > 1.0:  # CFL violation: shrink at once
            dt_safe = current_dt * config.shrink_factor
    dt_new = min(max(dt_safe, config.dt_min), config.dt_max)
    diagnostics = {
        "dt": float(dt_new),
        "dt_adv": float(dt_adv),
        "dt_diff": float(dt_diff),
        "cfl_adv": float(dt_new / dt_adv),
        "cfl_diff": float(dt_new / dt_diff) if dt_diff < math.inf else 0.0,
        "max_velocity": float(vmax),
        "limited_by": "advection" if dt_adv < dt_diff else "diffusion",
    }
    return float(dt_new), diagnostics


class AdaptiveTimestepper:
    """Adaptive step controller (adaptive_timestep.py:202-331)."""

    def __init__(self, grid, config: Optional[CFLConfig] = None, verbose: bool = False):
        self.grid = grid
        self.config = config or CFLConfig()
        self.verbose = verbose
        self.dt_history: list = []
        self.cfl_history: list = []
        self.time_history: list = []
        self.n_steps = 0
        self.n_rejected = 0
        self.n_dt_changes = 0

    def compute_timestep(self, state, u, v, nu_p: float = 0.0, p: int = 8, *,
                         max_velocity: Optional[float] = None):
        """Next step from (u, v), or from their maximum speed when the
        caller already has it (``max_velocity``; u and v are then unused)."""
        current_dt = self.dt_history[-1] if self.dt_history else None
        vmax = compute_max_velocity(u, v) if max_velocity is None else max_velocity
        dt_new, diags = timestep_from_speed(vmax, self.grid, self.config, nu_p, p, current_dt)
        if current_dt is not None and abs(dt_new / current_dt - 1.0) > 0.1:
            self.n_dt_changes += 1
            if self.verbose:
                print(f"Timestep change: {current_dt:.3e} -> {dt_new:.3e} (ratio {dt_new / current_dt:.2f})")
        self.dt_history.append(dt_new)
        self.cfl_history.append(diags["cfl_adv"])
        self.time_history.append(state.get("time", 0.0))
        self.n_steps += 1
        return dt_new, diags

    def check_stability(self, state_before, state_after, dt_used):
        """Non-finite values or a more than tenfold growth of max |theta_hat|
        reject the step (adaptive_timestep.py:276-305)."""
        after = state_after["theta_hat"]
        pl = _field_plan(after)
        m_after = pl.spectrum_absmax(pl.check_spectrum(after))
        if not math.isfinite(m_after):
            return False, "NaN or Inf detected"
        before = state_before["theta_hat"]
        m_before = pl.spectrum_absmax(pl.check_spectrum(before))
        growth = m_after / (m_before + 1e-10)
        if growth > 10.0:
            return False, f"Excessive growth: {growth:.2f}x"
        return True, None

    def suggest_retry_timestep(self, dt_failed: float) -> float:
        self.n_rejected += 1
        dt_retry = dt_failed * self.config.shrink_factor
        if self.verbose:
            print(f"Timestep rejected, retrying with dt={dt_retry:.3e}")
        return max(dt_retry, self.config.dt_min)

    def get_statistics(self) -> dict:
        if not self.dt_history:
            return {}
        dts, cfls = self.dt_history, self.cfl_history
        return {
            "n_steps": self.n_steps,
            "n_rejected": self.n_rejected,
            "n_dt_changes": self.n_dt_changes,
            "dt_min_used": min(dts),
            "dt_max_used": max(dts),
            "dt_mean": sum(dts) / len(dts),
            "cfl_mean": sum(cfls) / len(cfls),
            "cfl_max": max(cfls),
            "efficiency": 1.0 - self.n_rejected / (self.n_steps + self.n_rejected),
        }

    def reset_history(self):
        self.dt_history.clear()
        self.cfl_history.clear()
        self.time_history.clear()
        self.n_steps = 0
        self.n_rejected = 0
        self.n_dt_changes = 0


def estimate_initial_timestep(grid, nu_p: float = 0.0, p: int = 8, target_cfl: float = 0.5) -> float:
    """adaptive_timestep.py:334-377 (typical velocity 1)."""
    dx = grid.L / grid.N
    dt_adv = target_cfl * dx / 1.0
    if nu_p > 0:
        return min(dt_adv, compute_diffusion_cfl(grid, nu_p, p) * target_cfl)
    return dt_adv
