"""Run logging (mirrors pygsquig/utils/logging.py: SimulationLogger,
ProgressBar, setup_logging, get_logger; same message formats)."""

from __future__ import annotations

import json
import logging
import sys
from datetime import datetime
from pathlib import Path
from typing import Any, Optional


class SimulationLogger:
    """Console (and optional file) logger with structured extras
    (logging.py:15-153)."""

    def __init__(self, name: str = "pygsquig", console_level: str = "INFO", file_path: Optional[Path] = None,
                 file_level: str = "DEBUG"):
        self.logger = logging.getLogger(name)
        self.logger.setLevel(logging.DEBUG)
        self.logger.handlers = []
        con = logging.StreamHandler(sys.stdout)
        con.setLevel(getattr(logging, console_level.upper()))
        con.setFormatter(logging.Formatter("%(asctime)s | %(levelname)-8s | %(message)s", datefmt="%H:%M:%S"))
        self.logger.addHandler(con)
        if file_path:
            file_path = Path(file_path)
            file_path.parent.mkdir(parents=True, exist_ok=True)
            fh = logging.FileHandler(file_path)
            fh.setLevel(getattr(logging, file_level.upper()))
            fh.setFormatter(logging.Formatter("%(asctime)s | %(name)s | %(levelname)-8s | %(message)s"))
            self.logger.addHandler(fh)
        self.metadata: dict[str, Any] = {}

    def set_metadata(self, **kwargs):
        self.metadata.update(kwargs)

    def _fmt(self, message: str, kwargs) -> str:
        extra = {**self.metadata, **kwargs}
        return f"{message} | {json.dumps(extra, default=str)}" if extra else message

    def info(self, message: str, **kwargs):
        self.logger.info(self._fmt(message, kwargs))

    def debug(self, message: str, **kwargs):
        self.logger.debug(self._fmt(message, kwargs))

    def warning(self, message: str, **kwargs):
        self.logger.warning(self._fmt(message, kwargs))

    def error(self, message: str, **kwargs):
        self.logger.error(self._fmt(message, kwargs))

    def log_simulation_start(self, config, device: str = "cuda"):
        self.info("=" * 60)
        self.info("pygSQuiG Simulation Starting")
        self.info(f"Grid: {config.grid.N}×{config.grid.N}, L={config.grid.L:.3f}")
        self.info(f"Solver: α={config.solver.alpha}, ν_p={config.solver.dissipation.nu_p:.2e}")
        self.info(f"Time: t_end={config.simulation.t_end}")
        self.info(f"Device: {device}")
        if config.forcing:
            self.info(f"Forcing: k_f={config.forcing.kf}, ε={config.forcing.epsilon}")
        self.info("=" * 60)

    def log_progress(self, time: float, step: int, dt: float, diagnostics: dict, eta_seconds: Optional[float] = None):
        parts = [f"t={time:8.3f}", f"step={step:6d}", f"dt={dt:.2e}"]
        for key, label, fmt in (("theta_rms", "θ_rms", ".3e"), ("energy", "E", ".3e"),
                                ("enstrophy", "Ω", ".3e"), ("cfl", "CFL", ".3f")):
            if key in diagnostics:
                parts.append(f"{label}={diagnostics[key]:{fmt}}")
        if eta_seconds is not None and eta_seconds > 0:
            s = int(eta_seconds)
            parts.append(f"ETA={s // 3600:02d}:{(s % 3600) // 60:02d}:{s % 60:02d}")
        self.info(" | ".join(parts))

    def log_checkpoint(self, checkpoint_path: Path, time: float, step: int):
        self.info(f"Checkpoint saved: {Path(checkpoint_path).name}", time=time, step=step)

    def log_output(self, output_path: Path, time: float, step: int):
        self.debug(f"Output saved: {Path(output_path).name}", time=time, step=step)

    def log_simulation_complete(self, final_time: float, total_steps: int, wall_time: float):
        self.info("=" * 60)
        self.info("Simulation Complete!")
        self.info(f"Final time: {final_time:.3f}")
        self.info(f"Total steps: {total_steps}")
        self.info(f"Wall time: {wall_time:.1f} seconds")
        self.info(f"Performance: {total_steps / max(wall_time, 1e-12):.1f} steps/second")
        self.info("=" * 60)


class ProgressBar:
    """Text progress bar over simulated time (logging.py:156-185)."""

    def __init__(self, total: float, width: int = 50):
        self.total, self.width = total, width
        self.start = datetime.now()

    def update(self, current: float) -> str:
        frac = min(max(current / self.total, 0.0), 1.0) if self.total > 0 else 1.0
        n = int(self.width * frac)
        el = (datetime.now() - self.start).total_seconds()
        eta = el / frac - el if frac > 0 else 0.0
        return f"[{'█' * n}{'░' * (self.width - n)}] {frac * 100:5.1f}% | {el:.0f}s elapsed | ETA {eta:.0f}s"


def setup_logging(output_dir: Optional[Path] = None, console_level: str = "INFO",
                  file_level: str = "DEBUG") -> SimulationLogger:
    """Logger for a run; a timestamped file under <output_dir>/logs when
    output_dir is given (logging.py:188-215)."""
    log_file = None
    if output_dir:
        log_file = Path(output_dir) / "logs" / f"simulation_{datetime.now().strftime('%Y%m%d_%H%M%S')}.log"
    return SimulationLogger(console_level=console_level, file_path=log_file, file_level=file_level)


def get_logger(name: str = "pygsquig") -> logging.Logger:
    return logging.getLogger(name)
