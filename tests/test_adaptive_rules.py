"""Host-side rules of adaptive stepping (no GPU): CFLConfig validation, the
step-size rule given a maximum speed, the step controller's bookkeeping,
the initial estimate and the generic RK4 / SSP-RK3 integrators.

Mirrors the reference's tests/test_adaptive_timestep.py and
tests/test_time_integrator.py cases that need no velocity field; those that
do run on the GPU (test_gpu_adaptive.py).
"""

import math

import numpy as np
import pytest
import torch

from pygsquig_b200 import make_grid
from pygsquig_b200.core.adaptive_timestep import (
    AdaptiveTimestepper,
    CFLConfig,
    compute_diffusion_cfl,
    estimate_initial_timestep,
    timestep_from_speed,
)
from pygsquig_b200.core.time_integrator import compute_diffusion_timestep, rk4_step, ssp_rk3_step

G64 = make_grid(64, 2 * math.pi)


def test_default_config_valid():
    c = CFLConfig()
    assert 0 < c.cfl_safety <= 1 and c.dt_min < c.dt_max and c.growth_factor > 1 and 0 < c.shrink_factor < 1


@pytest.mark.parametrize("kw", [dict(cfl_safety=0.0), dict(cfl_safety=1.5), dict(dt_min=1.0, dt_max=0.1),
                                dict(growth_factor=0.9), dict(shrink_factor=1.0), dict(target_cfl=0.0)])
def test_invalid_config(kw):
    with pytest.raises(ValueError):
        CFLConfig(**kw)


def test_diffusion_limits():
    dx = G64.L / G64.N
    assert math.isclose(compute_diffusion_cfl(G64, 0.1, p=1), 0.25 * dx**2 / 0.1)
    d = compute_diffusion_cfl(G64, 1e-8, 4)
    kmax = math.pi * G64.N / G64.L
    assert math.isclose(d, dx**8 / (1e-8 * kmax**6)) and 0 < d < math.inf
    assert compute_diffusion_cfl(G64, 0.0, 2) == math.inf
    assert compute_diffusion_timestep(0.0, 10.0) == math.inf
    assert math.isclose(compute_diffusion_timestep(0.5, 100.0, 0.8), 0.8 * 2 / 50)


def test_advection_limited():
    c = CFLConfig()
    dt, d = timestep_from_speed(10.0, G64, c, nu_p=0.0, p=2)
    assert d["limited_by"] == "advection" and dt <= d["dt_adv"]
    assert 0 < d["cfl_adv"] <= c.cfl_safety
    assert math.isclose(d["dt_adv"], (G64.L / G64.N) / 10.0)


def test_diffusion_limited():
    dt, d = timestep_from_speed(0.1, G64, CFLConfig(), nu_p=1.0, p=1)
    assert d["limited_by"] == "diffusion" and dt <= d["dt_diff"]


def test_bounds_growth_and_shrink():
    c = CFLConfig(dt_min=1e-4, dt_max=1e-2)
    dt, _ = timestep_from_speed(1000.0, G64, c)
    assert c.dt_min <= dt <= c.dt_max
    c = CFLConfig(growth_factor=1.5)
    dt, _ = timestep_from_speed(0.1, G64, c, current_dt=1e-3)
    assert dt <= 1e-3 * 1.5
    c = CFLConfig(shrink_factor=0.5)
    safe, d = timestep_from_speed(10.0, G64, c)
    dt, _ = timestep_from_speed(10.0, G64, c, current_dt=safe * 2.0)
    assert dt < safe * 2.0
    assert math.isclose(dt, safe * 2.0 * 0.5)  # CFL number > 1: shrink at once


def test_properties_safety_and_monotonic():
    c = CFLConfig(cfl_safety=0.7)
    dts = []
    for vel in (0.1, 1.0, 10.0, 100.0):
        dt, d = timestep_from_speed(vel, G64, c)
        assert d["cfl_adv"] <= c.cfl_safety + 1e-10
        dts.append(dt)
    assert all(a >= b for a, b in zip(dts, dts[1:]))


def test_zero_speed_uses_floor():
    dt, d = timestep_from_speed(0.0, G64, CFLConfig())
    assert d["max_velocity"] == 0.0 and dt == CFLConfig().dt_max


def test_timestepper_bookkeeping():
    ts = AdaptiveTimestepper(make_grid(32, 2 * math.pi), CFLConfig())
    assert ts.n_steps == 0 and ts.n_rejected == 0 and not ts.dt_history and ts.get_statistics() == {}
    state = {"time": 0.0}
    for _ in range(5):
        dt, d = ts.compute_timestep(state, None, None, max_velocity=1.0)
        assert dt > 0 and "cfl_adv" in d
        state["time"] += 0.1
    st = ts.get_statistics()
    assert st["n_steps"] == 5 and st["efficiency"] == 1.0 and "dt_mean" in st and "cfl_mean" in st
    assert ts.suggest_retry_timestep(0.01) == 0.01 * ts.config.shrink_factor and ts.n_rejected == 1
    assert ts.get_statistics()["efficiency"] == 1.0 - 1 / 6
    assert ts.suggest_retry_timestep(1e-9) == ts.config.dt_min
    ts.reset_history()
    assert ts.n_steps == 0 and not ts.dt_history


def test_initial_estimate():
    g = make_grid(128, 2 * math.pi)
    a = estimate_initial_timestep(g, nu_p=0.0, target_cfl=0.5)
    assert 0 < a < 1.0 and math.isclose(a, 0.5 * g.L / g.N)
    assert estimate_initial_timestep(g, nu_p=0.01, p=2, target_cfl=0.5) <= estimate_initial_timestep(g, nu_p=0.0)


def test_rk4_and_ssp_rk3_linear_ode():
    """y' = lam y: one step equals the stability polynomial of each scheme."""
    lam, dt = -0.7 + 0.3j, 0.1
    y0 = torch.tensor([1.0 + 0.5j, -2.0 + 0j], dtype=torch.complex128)
    z = lam * dt
    y4 = rk4_step(y0, lambda y: lam * y, dt)
    y3 = ssp_rk3_step(y0, lambda y: lam * y, dt)
    np.testing.assert_allclose(y4.numpy(), (1 + z + z**2 / 2 + z**3 / 6 + z**4 / 24) * y0.numpy(), rtol=1e-14)
    np.testing.assert_allclose(y3.numpy(), (1 + z + z**2 / 2 + z**3 / 6) * y0.numpy(), rtol=1e-14)


def test_ssp_rk3_tvd():
    """First-order upwind advection with SSP-RK3 at CFL 1 does not increase
    total variation (time_integrator tests of the reference)."""
    n = 64
    x = torch.linspace(0, 1, n + 1, dtype=torch.float64)[:-1]
    u0 = (x > 0.3).double() * (x < 0.6).double()
    dx, c = 1.0 / n, 1.0
    rhs = lambda u: -c * (u - torch.roll(u, 1)) / dx  # noqa: E731
    tv = lambda u: float((u - torch.roll(u, 1)).abs().sum())  # noqa: E731
    u = u0
    for _ in range(20):
        u = ssp_rk3_step(u, rhs, 1.0 * dx / c)
        assert tv(u) <= tv(u0) + 1e-12
