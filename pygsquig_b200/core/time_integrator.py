"""Generic explicit integrators and step limits (mirrors pygsquig/core/time_integrator.py).

``rk4_step`` and ``ssp_rk3_step`` take any right-hand side on tensors (the
solver's own RK4 runs in the library's fused stage kernels; these serve
user-written right-hand sides, e.g. ``solver.compute_rhs``).  The step
limits reduce (N, N) fields on the device with the library's NaN-aware
max-speed reduction.
"""

from __future__ import annotations

import math
from typing import Any, Callable

import torch

from .adaptive_timestep import _field_plan


def rk4_step(state, rhs_fn: Callable[..., Any], dt: float, *args: Any):
    """Classical RK4 (time_integrator.py:14-36)."""
    k1 = rhs_fn(state, *args)
    k2 = rhs_fn(state + 0.5 * dt * k1, *args)
    k3 = rhs_fn(state + 0.5 * dt * k2, *args)
    k4 = rhs_fn(state + dt * k3, *args)
    return state + dt * (k1 + 2 * k2 + 2 * k3 + k4) / 6


def ssp_rk3_step(state, rhs_fn: Callable[..., Any], dt: float, *args: Any):
    """Shu-Osher three-stage SSP-RK3 (time_integrator.py:39-67)."""
    u1 = state + dt * rhs_fn(state, *args)
    u2 = 0.75 * state + 0.25 * u1 + 0.25 * dt * rhs_fn(u1, *args)
    return state / 3 + (2 / 3) * u2 + (2 / 3) * dt * rhs_fn(u2, *args)


def _absmax(x) -> float:
    """max |x| of an (N, N) field, reduced on the device."""
    pl = _field_plan(x)
    t = pl.check_real(x)
    return pl.max_speed(t, torch.zeros_like(t))


def compute_cfl(u, v, dx: float, dy: float, safety_factor: float = 0.8) -> float:
    """safety * min(dx / (pi max|u|), dy / (pi max|v|)) (time_integrator.py:70-100)."""
    u_max, v_max = _absmax(u), _absmax(v)
    dt_x = dx / (math.pi * u_max) if u_max > 0 else math.inf
    dt_y = dy / (math.pi * v_max) if v_max > 0 else math.inf
    return float(safety_factor * min(dt_x, dt_y))


def compute_diffusion_timestep(nu: float, k2_max: float, safety_factor: float = 0.8) -> float:
    """safety * 2 / (nu k2_max) (time_integrator.py:103-122)."""
    if nu <= 0 or k2_max <= 0:
        return math.inf
    return float(safety_factor * 2.0 / (nu * k2_max))


def adaptive_timestep(u, v, grid_dx: float, nu: float = 0.0, k2_max: float = 0.0, dt_max: float = 0.1,
                      cfl_safety: float = 0.8) -> float:
    """min(CFL, diffusion, dt_max) (time_integrator.py:125-160)."""
    dt = min(compute_cfl(u, v, grid_dx, grid_dx, cfl_safety), compute_diffusion_timestep(nu, k2_max, cfl_safety))
    if dt_max is not None:
        dt = min(dt, dt_max)
    return float(dt)
