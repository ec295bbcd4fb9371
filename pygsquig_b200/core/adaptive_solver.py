"""gSQG solver with CFL-adaptive steps (mirrors pygsquig/core/adaptive_solver.py).

Each step reads one number back from the device (the maximum speed) to
choose dt, runs the library's RK4 step and checks the result with the
NaN-aware max |theta_hat| reduction; a rejected step is retried once from
the saved state at the shrunk dt, as the reference does.
"""

from __future__ import annotations

import time as pytime
from typing import Any, Callable, Optional

from .adaptive_timestep import AdaptiveTimestepper, CFLConfig, estimate_initial_timestep, timestep_from_speed
from .solver import State, gSQGSolver


class AdaptivegSQGSolver:
    """adaptive_solver.py:22-343.  ``precision`` and ``scheme`` select the
    base solver's arithmetic and integrator (extensions; the defaults are
    the reference's FP64 explicit RK4)."""

    def __init__(self, grid, alpha: float, nu_p: float = 0.0, p: int = 8,
                 cfl_config: Optional[CFLConfig] = None, verbose: bool = False, *,
                 precision: str = "float64", scheme: str = "explicit"):
        self.base_solver = gSQGSolver(grid, alpha, nu_p, p, precision=precision, scheme=scheme)
        self.grid = grid
        self.alpha = alpha
        self.nu_p = nu_p
        self.p = p
        self.verbose = verbose
        self.timestepper = AdaptiveTimestepper(grid, cfl_config, verbose=verbose)
        self.current_dt = estimate_initial_timestep(
            grid, nu_p, p, target_cfl=cfl_config.target_cfl if cfl_config else 0.5)
        if verbose:
            print(f"Initial timestep estimate: {self.current_dt:.3e}")

    def initialize(self, **kwargs) -> State:
        return self.base_solver.initialize(**kwargs)

    def _max_speed(self, theta_hat) -> float:
        pl = self.base_solver.aux_plan()
        u, v = pl.velocity(pl.check_spectrum(theta_hat))
        return pl.max_speed(u, v)

    def step(self, state: State, forcing: Optional[Callable] = None, damping: Optional[Callable] = None,
             dt_max: Optional[float] = None, **kwargs) -> tuple[State, dict[str, Any]]:
        """One adaptive step with one retry (adaptive_solver.py:81-165)."""
        vmax = self._max_speed(state["theta_hat"])
        dt, dt_diags = self.timestepper.compute_timestep(state, None, None, self.nu_p, self.p, max_velocity=vmax)
        if dt_max is not None:
            dt = min(dt, dt_max)
        state_backup = dict(state)
        try:
            new_state = self.base_solver.step(state, dt, forcing=forcing, damping=damping, **kwargs)
            ok, reason = self.timestepper.check_stability(state, new_state, dt)
            if not ok:
                if self.verbose:
                    print(f"Step rejected: {reason}")
                dt = self.timestepper.suggest_retry_timestep(dt)
                new_state = self.base_solver.step(state_backup, dt, forcing=forcing, damping=damping, **kwargs)
                dt_diags["retry"] = True
        except Exception as e:  # the reference retries any failure of the step once
            if self.verbose:
                print(f"Step failed with error: {e}")
            dt = self.timestepper.suggest_retry_timestep(dt)
            new_state = self.base_solver.step(state_backup, dt, forcing=forcing, damping=damping, **kwargs)
            dt_diags["retry"] = True
            dt_diags["error"] = str(e)
        self.current_dt = dt
        return new_state, {"dt_used": dt, "dt_diagnostics": dt_diags, "time": new_state["time"],
                           "step": new_state["step"]}

    def evolve(self, state: State, t_final: float, forcing: Optional[Callable] = None,
               damping: Optional[Callable] = None, save_interval: Optional[float] = None,
               callback: Optional[Callable] = None, max_steps: int = 100000, min_progress_rate: float = 1e-6,
               **kwargs) -> dict[str, Any]:
        """Adaptive steps up to t_final (adaptive_solver.py:167-318): the last
        step and each save time are hit exactly, a step budget and a minimum
        simulated-time-per-wall-second rate stop runs that stall."""
        results: dict[str, Any] = {"times": [], "states": [], "dt_history": [], "diagnostics": []}
        wall0 = pytime.perf_counter()
        t0 = state["time"]
        last_check = wall0
        if save_interval is not None:
            results["times"].append(state["time"])
            results["states"].append(dict(state))
            next_save = state["time"] + save_interval
        else:
            next_save = t_final + 1
        cur, n, last_dt = state, 0, None
        if self.verbose:
            print(f"Evolving from t={state['time']} to t={t_final}")
        while cur["time"] < t_final:
            if n >= max_steps:
                raise RuntimeError(
                    f"Maximum steps ({max_steps}) reached. Current time: {cur['time']:.6f}, "
                    f"Target: {t_final:.6f}, Last dt: {last_dt if last_dt is not None else 'N/A'}")
            now = pytime.perf_counter()
            if now - last_check > 1.0:
                elapsed, progress = now - wall0, cur["time"] - t0
                if elapsed > 0 and progress / elapsed < min_progress_rate:
                    raise RuntimeError(
                        f"Progress too slow. Rate: {progress / elapsed:.2e} < {min_progress_rate:.2e}. "
                        f"Simulated {progress:.6f} in {elapsed:.1f}s")
                last_check = now
            dt_max = t_final - cur["time"]
            if save_interval is not None:
                dt_max = min(dt_max, next_save - cur["time"])
            new, info = self.step(cur, forcing=forcing, damping=damping, dt_max=dt_max, **kwargs)
            if new["time"] <= cur["time"]:
                raise RuntimeError(f"Time not advancing: dt={info['dt_used']}, time={cur['time']}")
            cur, n, last_dt = new, n + 1, info["dt_used"]
            if save_interval is not None and cur["time"] >= next_save:
                results["times"].append(cur["time"])
                results["states"].append(dict(cur))
                results["dt_history"].append(info["dt_used"])
                results["diagnostics"].append(info["dt_diagnostics"])
                next_save += save_interval
            if callback is not None:
                callback(cur, info)
            if self.verbose and n % 100 == 0:
                frac = (cur["time"] - t0) / (t_final - t0)
                el = pytime.perf_counter() - wall0
                print(f"  Step {n}: t={cur['time']:.3f} ({frac * 100:.1f}%), dt={info['dt_used']:.3e}, "
                      f"CFL={info['dt_diagnostics']['cfl_adv']:.3f}, ETA={el / frac - el if frac > 0 else 0:.1f}s")
        if save_interval is not None and cur["time"] > results["times"][-1]:
            results["times"].append(cur["time"])
            results["states"].append(dict(cur))
        wall = pytime.perf_counter() - wall0
        stats = self.timestepper.get_statistics()
        stats["total_steps"] = n
        stats["wall_time"] = wall
        stats["simulated_time"] = cur["time"] - state["time"]
        stats["time_ratio"] = stats["simulated_time"] / wall
        results["statistics"] = stats
        results["final_state"] = cur
        if self.verbose:
            print(f"\nEvolution complete:\n  Total steps: {n}\n  Wall time: {wall:.2f}s")
            if "dt_mean" in stats:
                print(f"  Mean timestep: {stats['dt_mean']:.3e}\n  Efficiency: {stats['efficiency'] * 100:.1f}%")
        return results

    def get_diagnostics(self, state: State) -> dict[str, float]:
        """Base diagnostics plus the CFL numbers of the step that would be
        taken now (adaptive_solver.py:320-343).  Unlike the reference this
        does not append to the stepper's history."""
        diags = self.base_solver.get_diagnostics(state)
        cur = self.timestepper.dt_history[-1] if self.timestepper.dt_history else None
        _, d = timestep_from_speed(self._max_speed(state["theta_hat"]), self.grid, self.timestepper.config,
                                   self.nu_p, self.p, cur)
        diags.update({f"cfl_{k}": v for k, v in d.items() if k.startswith("cfl_")})
        diags["current_dt"] = self.current_dt
        diags["max_velocity"] = d["max_velocity"]
        return diags
