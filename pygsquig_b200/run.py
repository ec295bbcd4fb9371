"""Run a simulation from a YAML configuration (mirrors pygsquig/scripts/run.py).

    python -m pygsquig_b200.run config.yml [--checkpoint FILE] [--output-dir DIR]
                                           [--dry-run] [--log-level LEVEL]
                                           [--precision float64|float32] [--scheme explicit|ifrk4]

Same configuration file, directory layout (checkpoints/, fields/,
diagnostics/, logs/, config.yml), event rules (log, output and checkpoint
intervals measured in simulated time, wall-time limit, Ctrl+C saves and
exits) and final files as the reference's driver.

Differences that come from running on the GPU:

* Fixed-step runs advance in segments: the steps up to the next log, output
  or checkpoint event go to ``solver.multistep`` (one CUDA-graph replay per
  step, ring phases for the whole segment uploaded once) instead of one
  Python call per step.  Simulated time is accumulated step by step on the
  host exactly as a per-step loop would, so events fire on the same steps.
* Ring phases come from ``numpy.random.default_rng(forcing.seed or 42)``
  (the reference draws them with jax.random).
* Files are HDF5 when h5py is installed, else ``.npz`` archives with the
  same layout; field outputs are ``.npz`` (the reference writes NetCDF
  through xarray, which is not a dependency here).
* Scalar sources other than ``none`` are rejected: the GPU scalar stages
  support none or a mean-gradient source.
"""

from __future__ import annotations

import logging
import math
import signal
import time
from pathlib import Path

import click
import numpy as np
import torch

from .core.grid import ifft2, make_grid
from .core.solver import gSQGSolver
from .core.solver_with_scalars import gSQGSolverWithScalars
from .core.time_integrator import adaptive_timestep
from .forcing import CombinedDamping, RingForcing
from .io import load_checkpoint, load_config, save_checkpoint, save_diagnostics, save_output
from .io.checkpoint import h5py
from .utils.diagnostics import compute_enstrophy, compute_total_energy
from .utils.runlog import RunLog

_shutdown = {"requested": False}


def _on_sigint(signum, frame):
    _shutdown["requested"] = True


def _ext(kind: str) -> str:
    if kind == "fields":
        return ".npz"
    return ".h5" if h5py is not None else ".npz"


def setup_output_directories(output_dir: Path, config, logger) -> dict:
    """run.py:36-57."""
    output_dir.mkdir(parents=True, exist_ok=True)
    dirs = {k: output_dir / k for k in ("checkpoints", "fields", "diagnostics")}
    for d in dirs.values():
        d.mkdir(exist_ok=True)
    config.to_yaml(output_dir / "config.yml")
    logger.event("config", file=str(output_dir / "config.yml"))
    return dirs


def create_source_from_config(source_config):
    """run.py:60-86 accepts exponential / localized / chemical / periodic;
    the GPU scalar stages carry no such source."""
    if source_config is None or source_config.type == "none":
        return None
    raise NotImplementedError(
        f"scalar source '{source_config.type}' is not supported by the GPU scalar stages "
        "(supported: none, or MeanGradientSource through the Python API)")


def _scalar_field(species, grid, seed):
    N, p = grid.N, species.initial_params
    ic = species.initial_condition
    if ic == "random":
        rng = np.random.default_rng(p.get("seed", (seed or 0) + 1))
        return p.get("amplitude", 1.0) * rng.standard_normal((N, N))
    if ic == "uniform":
        return p.get("value", 1.0) * np.ones((N, N))
    if ic == "gaussian":
        x0, y0 = p.get("center", [grid.L / 2, grid.L / 2])
        w = p.get("width", 1.0)
        x, y = grid.x.cpu().numpy(), grid.y.cpu().numpy()
        return np.exp(-((x - x0) ** 2 + (y - y0) ** 2) / (2 * w**2))
    return np.zeros((N, N))


def initialize_simulation(config, checkpoint_path, logger, precision="float64", scheme="explicit"):
    """run.py:89-193: grid, solver and the initial state (from a checkpoint,
    a seeded random field or zero)."""
    grid = make_grid(config.grid.N, config.grid.L)
    kw = dict(precision=precision, scheme=scheme)
    sc = config.solver
    if config.scalars and config.scalars.enabled:
        species = {s.name: {"kappa": s.kappa, "source": create_source_from_config(s.source)}
                   for s in config.scalars.species}
        solver = gSQGSolverWithScalars(grid, sc.alpha, sc.dissipation.nu_p, sc.dissipation.p,
                                       passive_scalars=species, **kw)
        logger.event("solver", alpha=sc.alpha, scalars=len(species), precision=precision, scheme=scheme)
    else:
        solver = gSQGSolver(grid, sc.alpha, sc.dissipation.nu_p, sc.dissipation.p, **kw)
    ic = config.initial_condition
    if checkpoint_path is None and ic.type == "checkpoint":
        checkpoint_path = ic.checkpoint_path
    if checkpoint_path:
        state, _ = load_checkpoint(checkpoint_path)
        state["theta_hat"] = state["theta_hat"].to(solver.cdtype).cuda()
        logger.event("resume", file=str(checkpoint_path), t=float(state["time"]), step=int(state["step"]))
        return grid, solver, state
    scal = None
    if config.scalars and config.scalars.enabled:
        scal = {s.name: _scalar_field(s, grid, ic.seed) for s in config.scalars.species}
    if ic.type == "random":
        kw0 = dict(seed=ic.seed)
    elif ic.type == "zero":
        kw0 = dict(theta0=np.zeros((grid.N, grid.N)))
    else:
        raise NotImplementedError(f"Initial condition type '{ic.type}' not implemented")
    state = solver.initialize(scalar_init=scal, **kw0) if scal is not None else solver.initialize(**kw0)
    logger.event("initial", kind=ic.type, seed=ic.seed, scalars=len(scal) if scal else 0)
    return grid, solver, state


def compute_streamfunction(theta_hat, grid, alpha: float):
    """psi_hat = |k|^-alpha theta_hat, zero at k = 0 (operators.py:134-155)."""
    k2 = grid.k2.to(theta_hat.device)
    op = torch.where(k2 > 0, torch.where(k2 > 0, k2, torch.ones_like(k2)).sqrt() ** (-alpha), torch.zeros_like(k2))
    return op.to(theta_hat.dtype) * theta_hat


def compute_diagnostics(state, grid, solver) -> dict:
    """run.py:196-227."""
    th_hat = state["theta_hat"]
    theta = ifft2(th_hat)
    d = {"theta_rms": float(torch.sqrt(torch.mean(theta.double() ** 2))),
         "theta_max": float(theta.abs().max()),
         "energy": compute_total_energy(th_hat, grid, solver.alpha),
         "enstrophy": compute_enstrophy(th_hat, grid, solver.alpha)}
    d.update(solver.get_diagnostics({k: v for k, v in state.items() if k != "scalar_state"}))
    return d


def _fields(state, grid, config, logger, solver):
    data = {}
    th_hat = state["theta_hat"]
    for f in config.output.fields:
        if f == "theta":
            data["theta"] = ifft2(th_hat)
        elif f == "vorticity":
            logger.event("skip_field", logging.WARNING, field="vorticity", why="not produced by this driver")
        elif f == "streamfunction":
            data["streamfunction"] = ifft2(compute_streamfunction(th_hat, grid, config.solver.alpha))
        elif f == "velocity":
            data["u"], data["v"] = solver.compute_velocity(th_hat)
        elif f == "scalars" and state.get("scalar_state") is not None:
            for name, sh in state["scalar_state"].scalars.items():
                data[f"scalar_{name}"] = ifft2(sh)
    return data


class Driver:
    """The time loop of run.py:299-530 with fixed-step segments on the GPU."""

    def __init__(self, config, grid, solver, state, dirs, logger):
        self.cfg, self.grid, self.solver, self.state = config, grid, solver, state
        self.dirs, self.log = dirs, logger
        fc = config.forcing
        self.ring = None
        if fc and fc.type == "ring":
            self.ring = RingForcing(kf=fc.kf, dk=fc.dk, epsilon=fc.epsilon, tau_f=fc.tau_f)
            self.rng = np.random.default_rng(fc.seed if fc.seed else 42)
            self.n_ring = self.ring.n_modes(grid)
            logger.event("forcing", kind="ring", kf=fc.kf, dk=fc.dk, eps=fc.epsilon, tau_f=fc.tau_f)
        self.damping = None
        dc = config.solver.damping
        if dc and dc.type != "none":
            # the reference's driver damps with CombinedDamping(mu, kf, nu_p, p): drag below kf plus
            # a second hyperviscous term on top of the solver's own
            self.damping = CombinedDamping(mu=dc.mu, kf=fc.kf if fc else 20.0,
                                           nu_p=config.solver.dissipation.nu_p, p=config.solver.dissipation.p)
            logger.event("damping", mu=dc.mu, kf=fc.kf if fc else 20.0, nu_p=config.solver.dissipation.nu_p)

    # -- one adaptive or clamped step --
    def _dt(self) -> float:
        ti = self.cfg.solver.time_integration
        if not ti.adaptive_cfl:
            return ti.dt
        u, v = self.solver.compute_velocity(self.state["theta_hat"])
        dx = self.grid.L / self.grid.N
        # run.py:307-316 passes (dx, dy, cfl_safety, dt_max) positionally into
        # adaptive_timestep(u, v, grid_dx, nu, k2_max, dt_max, cfl_safety): dy lands in nu,
        # cfl_safety in k2_max and the CFL factor stays at its default 0.8.  Same call here,
        # so the steps are the reference's.
        return adaptive_timestep(u, v, dx, dx, ti.cfl_safety, ti.dt_max)

    def _forcing(self, dt):
        if self.ring is None:
            return None
        return self.ring.bind(self.rng.uniform(0, 2 * math.pi, self.n_ring), dt, self.grid)

    def _advance(self, n: int, dt: float, t_end_time: float):
        """n steps of size dt; time accumulated by repeated addition."""
        st = self.state
        if n == 1 or getattr(self.solver, "species", None):  # scalar runs step one at a time
            for _ in range(n):
                st = self.solver.step(st, dt, forcing=self._forcing(dt), damping=self.damping)
            self.state = st
            return
        noise = None if self.ring is None else self.rng.uniform(0, 2 * math.pi, (n, self.n_ring))
        new = self.solver.multistep(st, n, dt, forcing=self.ring, damping=self.damping, noise=noise)
        new["time"] = t_end_time
        self.state = new

    def run(self, t_start_wall):
        cfg, sim = self.cfg, self.cfg.simulation
        t_end = sim.t_end
        t0 = self.state["time"]
        last_out = last_ckpt = last_log = t0
        while self.state["time"] < t_end and not _shutdown["requested"]:
            dt = min(self._dt(), t_end - self.state["time"])
            if cfg.solver.time_integration.adaptive_cfl or dt != cfg.solver.time_integration.dt:
                self._advance(1, dt, self.state["time"] + dt)
            else:
                # steps until an event fires or dt would be clamped
                t, n = self.state["time"], 0
                while True:
                    t += dt
                    n += 1
                    if (t >= t_end or t - last_log >= sim.log_interval or t - last_out >= sim.output_interval
                            or t - last_ckpt >= sim.checkpoint_interval or min(dt, t_end - t) != dt):
                        break
                self._advance(n, dt, t)
            now = self.state["time"]
            if now - last_log >= sim.log_interval:
                d = compute_diagnostics(self.state, self.grid, self.solver)
                el = time.time() - t_start_wall
                rate = (now - last_log) / (time.time() - t_start_wall + el) if now > last_log else 0
                eta = (t_end - now) / rate if rate > 0 else None
                self.log.progress(now, self.state["step"], dt, d, eta)
                save_diagnostics(d, now, self.dirs["diagnostics"] / ("timeseries" + _ext("diag")))
                last_log = now
            if now - last_out >= sim.output_interval:
                step = self.state["step"]
                f = self.dirs["fields"] / f"fields_{step:08d}{_ext('fields')}"
                meta = {"step": int(step), "alpha": float(cfg.solver.alpha),
                        "nu_p": float(cfg.solver.dissipation.nu_p), "p": int(cfg.solver.dissipation.p)}
                save_output(_fields(self.state, self.grid, cfg, self.log, self.solver), self.grid, now, meta, f,
                            compress=cfg.output.compress)
                self.log.wrote("fields", f, now, step)
                last_out = now
            if now - last_ckpt >= sim.checkpoint_interval:
                step = self.state["step"]
                f = self.dirs["checkpoints"] / f"step_{step:08d}{_ext('ckpt')}"
                save_checkpoint(self.state, cfg, f)
                self.log.wrote("checkpoint", f, now, step)
                last_ckpt = now
            if sim.wall_time_limit and time.time() - t_start_wall > sim.wall_time_limit:
                self.log.event("wall_limit", logging.WARNING, limit_s=sim.wall_time_limit)
                _shutdown["requested"] = True
        return last_out


def run(config_path, checkpoint=None, output_dir="./output", dry_run=False, log_level="INFO",
        precision="float64", scheme="explicit"):
    cfg = load_config(config_path)
    out = Path(output_dir)
    if not dry_run:
        out.mkdir(parents=True, exist_ok=True)
    logger = RunLog(out if not dry_run else None, level=log_level)
    logger.event("config", file=str(config_path), N=cfg.grid.N, L=cfg.grid.L, alpha=cfg.solver.alpha,
                 t_end=cfg.simulation.t_end, dry_run=bool(dry_run))
    if dry_run:
        return None
    if not torch.cuda.is_available():
        raise RuntimeError("pygsquig_b200.run needs a CUDA device (the solver has no CPU path)")
    dirs = setup_output_directories(out, cfg, logger)
    _shutdown["requested"] = False
    old = signal.signal(signal.SIGINT, _on_sigint)
    try:
        grid, solver, state = initialize_simulation(cfg, checkpoint, logger, precision, scheme)
        logger.started(cfg, f"cuda ({torch.cuda.get_device_name()})")
        t_wall = time.time()
        drv = Driver(cfg, grid, solver, state, dirs, logger)
        last_out = drv.run(t_wall)
        state = drv.state
        step, now = state["step"], state["time"]
        f = dirs["checkpoints"] / f"final_step_{step:08d}{_ext('ckpt')}"
        save_checkpoint(state, cfg, f)
        logger.wrote("checkpoint", f, now, step)
        if now - last_out > 0:
            data = {"theta": ifft2(state["theta_hat"])}
            if state.get("scalar_state") is not None:
                for name, sh in state["scalar_state"].scalars.items():
                    data[f"scalar_{name}"] = ifft2(sh)
            f = dirs["fields"] / f"fields_final_{step:08d}{_ext('fields')}"
            save_output(data, grid, now, {"step": int(step)}, f)
            logger.wrote("fields", f, now, step)
        logger.finished(now, step, time.time() - t_wall)
        return state
    finally:
        signal.signal(signal.SIGINT, old)


@click.command()
@click.argument("config", type=click.Path(exists=True))
@click.option("--device", type=click.Choice(["gpu", "cuda"]), default="gpu", help="Device to run on (CUDA only)")
@click.option("--checkpoint", type=click.Path(exists=True), help="Path to checkpoint file to resume from")
@click.option("--output-dir", type=click.Path(), default="./output", help="Directory for output files")
@click.option("--dry-run", is_flag=True, help="Validate configuration without running")
@click.option("--log-level", type=click.Choice(["DEBUG", "INFO", "WARNING", "ERROR"]), default="INFO")
@click.option("--precision", type=click.Choice(["float64", "float32"]), default="float64")
@click.option("--scheme", type=click.Choice(["explicit", "ifrk4"]), default="explicit")
def main(config, device, checkpoint, output_dir, dry_run, log_level, precision, scheme):
    """Run a pygSQuiG simulation from a YAML configuration file."""
    run(config, checkpoint, output_dir, dry_run, log_level, precision, scheme)


if __name__ == "__main__":
    main()
