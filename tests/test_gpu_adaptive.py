"""Adaptive stepping on the GPU: the device max-speed and max-|theta_hat|
reductions (including NaN propagation) against numpy, and the adaptive
solver's step / evolve / retry behaviour, following the reference's
tests/test_adaptive_timestep.py.
"""

import math

import numpy as np
import pytest
import torch

from pygsquig_b200 import gSQGSolver, make_grid
from pygsquig_b200.core.adaptive_solver import AdaptivegSQGSolver
from pygsquig_b200.core.adaptive_timestep import (
    AdaptiveTimestepper,
    CFLConfig,
    compute_advection_cfl,
    compute_max_velocity,
    compute_timestep,
)
from pygsquig_b200.core.time_integrator import adaptive_timestep, compute_cfl

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    from pygsquig_b200.build import build

    build()


@pytest.mark.parametrize("N,dtype", [(64, torch.float64), (512, torch.float32), (2048, torch.float64)])
def test_max_speed_matches_numpy(N, dtype):
    g = torch.Generator().manual_seed(N)
    u = torch.randn(N, N, generator=g, dtype=torch.float64) * 3
    v = torch.randn(N, N, generator=g, dtype=torch.float64)
    u[N // 3, N // 5] = 40.0  # a unique maximum off the diagonal
    ref = float(np.sqrt(u.numpy() ** 2 + v.numpy() ** 2).max())
    got = compute_max_velocity(u.to(dtype).cuda(), v.to(dtype).cuda())
    tol = 1e-15 if dtype == torch.float64 else 1e-6
    assert abs(got - ref) <= tol * ref


def test_reference_velocity_cases():
    N, dx = 64, 2 * math.pi / 64
    z = torch.zeros(N, N, dtype=torch.float64)
    assert compute_max_velocity(z, z) == 0.0
    assert math.isclose(compute_max_velocity(z + 1, z + 1), math.sqrt(2), rel_tol=1e-15)
    assert math.isclose(compute_advection_cfl(z + 2, z, dx), dx / 2.0, rel_tol=1e-15)
    assert math.isclose(compute_cfl(z + 2, z - 4, dx, dx), 0.8 * dx / (math.pi * 4), rel_tol=1e-15)
    assert compute_cfl(z, z, dx, dx) == math.inf
    assert adaptive_timestep(z + 2, z, dx, dt_max=1e-9) == 1e-9
    u = z.clone()
    u[0, 0] = 0.1
    dt, d = compute_timestep(u, z, make_grid(N, 2 * math.pi), CFLConfig(), nu_p=1.0, p=1)
    assert d["limited_by"] == "diffusion" and dt <= d["dt_diff"]


def test_nan_propagates():
    N = 128
    u = torch.ones(N, N, dtype=torch.float32, device="cuda")
    u[7, 100] = float("nan")
    assert math.isnan(compute_max_velocity(u, torch.zeros_like(u)))
    ts = AdaptiveTimestepper(make_grid(N, 2 * math.pi))
    before = {"theta_hat": torch.ones(N, N, dtype=torch.complex128)}
    ok, why = ts.check_stability(before, {"theta_hat": before["theta_hat"] * 1.1}, 0.01)
    assert ok and why is None
    bad = before["theta_hat"].clone()
    bad[3, 4] = complex(float("nan"), 0.0)
    ok, why = ts.check_stability(before, {"theta_hat": bad}, 0.01)
    assert not ok and "NaN" in why
    bad[3, 4] = complex(0.0, float("inf"))
    ok, why = ts.check_stability(before, {"theta_hat": bad}, 0.01)
    assert not ok and "NaN" in why
    ok, why = ts.check_stability(before, {"theta_hat": before["theta_hat"] * 20.0}, 0.01)
    assert not ok and "growth" in why.lower()


def test_spectrum_absmax_matches_numpy():
    N = 1024
    rng = np.random.default_rng(5)
    th = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    th[900, 17] = 50 - 60j
    ts = AdaptiveTimestepper(make_grid(N, 2 * math.pi))
    from pygsquig_b200.core.adaptive_timestep import _field_plan

    for t in (torch.as_tensor(th), torch.as_tensor(th).to(torch.complex64)):
        pl = _field_plan(t)
        got = pl.spectrum_absmax(pl.check_spectrum(t))
        assert abs(got - abs(50 - 60j)) <= (1e-15 if t.dtype == torch.complex128 else 1e-6) * 78.2
    assert ts.check_stability({"theta_hat": th}, {"theta_hat": th * 2}, 0.1)[0]


def _smooth_ic(g):
    x, y = g.x.cpu().numpy(), g.y.cpu().numpy()
    return np.sin(2 * np.pi * x / g.L) * np.cos(2 * np.pi * y / g.L)


def test_single_step_and_diagnostics():
    g = make_grid(32, 2 * math.pi)
    s = AdaptivegSQGSolver(g, alpha=1.0, nu_p=1e-4, p=4)
    assert s.current_dt > 0 and hasattr(s, "timestepper")
    st = s.initialize(seed=42)
    new, info = s.step(st)
    assert new["time"] > st["time"] and info["dt_diagnostics"]["cfl_adv"] > 0
    # the chosen dt is the reference's rule applied to the velocity of theta_hat
    u, v = s.base_solver.compute_velocity(st["theta_hat"])
    vmax = float(torch.sqrt(u.double() ** 2 + v.double() ** 2).max())
    assert math.isclose(info["dt_diagnostics"]["max_velocity"], vmax, rel_tol=1e-13)
    ref = gSQGSolver(g, 1.0, 1e-4, 4).step(st, info["dt_used"])
    assert torch.equal(new["theta_hat"], ref["theta_hat"])
    d = s.get_diagnostics(new)
    assert d["current_dt"] == info["dt_used"] and d["max_velocity"] > 0 and "cfl_cfl_adv" in d


def test_evolve_to_target_and_vs_fixed():
    g = make_grid(32, 2 * math.pi)
    cfg = CFLConfig(cfl_safety=0.3, dt_max=0.01, dt_min=1e-6, target_cfl=0.3)
    s = AdaptivegSQGSolver(g, alpha=1.0, nu_p=1e-2, p=2, cfl_config=cfg)
    st = s.initialize(theta0=_smooth_ic(g))
    res = s.evolve(st, 0.05, save_interval=0.025, max_steps=10000, min_progress_rate=1e-4)
    assert res["final_state"]["time"] >= 0.05 - 1e-10
    assert len(res["times"]) >= 2 and 0 < res["statistics"]["total_steps"] < 10000
    assert all(abs(t - 0.025 * i) < 1e-12 for i, t in enumerate(res["times"][:3]))
    # adaptive vs a fixed dt = 1e-3 to t = 0.02 (reference: within 20 %; both are RK4 on a smooth field)
    s2 = AdaptivegSQGSolver(g, alpha=1.0, nu_p=1e-2, p=2, cfl_config=cfg)
    ra = s2.evolve(s2.initialize(theta0=_smooth_ic(g)), 0.02, max_steps=5000, min_progress_rate=1e-4)
    f = gSQGSolver(g, 1.0, 1e-2, 2)
    sf = f.initialize(theta0=_smooth_ic(g))
    for _ in range(20):
        sf = f.step(sf, 1e-3)
    a, b = ra["final_state"]["theta_hat"], sf["theta_hat"]
    assert float(torch.linalg.norm(a - b) / torch.linalg.norm(b)) < 1e-6


def test_retry_on_rejected_step():
    """A step the stability check rejects is redone from the saved state at
    the shrunk dt (adaptive_solver.py:121-139)."""
    g = make_grid(64, 2 * math.pi)
    s = AdaptivegSQGSolver(g, alpha=1.0, nu_p=0.0, p=8)
    st = s.initialize(seed=3)
    calls = []
    orig = s.timestepper.check_stability

    def reject_first(a, b, dt):
        calls.append(dt)
        return (False, "Excessive growth: planted") if len(calls) == 1 else orig(a, b, dt)

    s.timestepper.check_stability = reject_first
    new, info = s.step(st)
    assert info["dt_diagnostics"]["retry"] and s.timestepper.n_rejected == 1
    assert math.isclose(info["dt_used"], calls[0] * s.timestepper.config.shrink_factor)
    ref = gSQGSolver(g, 1.0, 0.0, 8).step(st, info["dt_used"])
    assert torch.equal(new["theta_hat"], ref["theta_hat"])


def test_evolve_stall_guards():
    g = make_grid(32, 2 * math.pi)
    s = AdaptivegSQGSolver(g, alpha=1.0, nu_p=1e-2, p=2, cfl_config=CFLConfig(dt_max=1e-4, dt_min=1e-8))
    with pytest.raises(RuntimeError, match="Maximum steps"):
        s.evolve(s.initialize(theta0=_smooth_ic(g)), 1.0, max_steps=5)


def test_forced_evolve_fp32():
    """Ring-forced FP32 run through evolve (no hyperviscosity: the reference's
    diffusion limit dx^(2p) / (nu k_max^(2p-2)) pins p = 8 runs to dt_min)."""
    from pygsquig_b200 import RingForcing

    g = make_grid(256, 2 * math.pi)
    s = AdaptivegSQGSolver(g, alpha=1.0, nu_p=0.0, p=8, precision="float32",
                           cfl_config=CFLConfig(dt_max=5e-3))
    ring = RingForcing(kf=20.0, dk=2.0, epsilon=0.1)
    st = s.initialize(seed=1)
    rng = np.random.default_rng(0)
    seen = []
    res = s.evolve(st, 0.05, forcing=ring, key=rng.uniform(0, 2 * math.pi, ring.n_modes(g)),
                   callback=lambda c, i: seen.append(i["dt_used"]))
    fin = res["final_state"]
    assert abs(fin["time"] - 0.05) < 1e-12 and bool(torch.isfinite(torch.view_as_real(fin["theta_hat"])).all())
    assert max(seen) <= 5e-3 and res["statistics"]["n_rejected"] == 0


@pytest.mark.parametrize("name", ["rk4_step", "ssp_rk3_step"])
def test_generic_integrators_on_device_rhs(name):
    """time_integrator.rk4_step / ssp_rk3_step driven by the library's RHS
    (solver.compute_rhs) match the float64 oracle's integrators on its RHS."""
    from oracle import sqg_oracle as O
    from pygsquig_b200.core import time_integrator as TI

    N, alpha, nu, p, dt = 64, 1.0, 1e-10, 8, 2e-3
    g = make_grid(N, 2 * math.pi)
    s = gSQGSolver(g, alpha, nu, p)
    th = s.initialize(seed=11)["theta_hat"]
    og = O.make_grid(N, 2 * math.pi)
    ref = th.cpu().numpy()
    got = th
    for _ in range(5):
        got = getattr(TI, name)(got, s.compute_rhs, dt)
        ref = getattr(O, name)(ref, lambda t: O.core_rhs(t, og, alpha, nu, p), dt)
    err = np.linalg.norm(got.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err < 1e-12, err
