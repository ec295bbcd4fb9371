"""Log of a driver run: one ``logging.Logger`` with key=value records.

Each record is one line, ``<elapsed> <level> <event> key=value ...``, written
to stdout and, for runs with an output directory, appended to
``<output>/logs/run.log``.  Events are short names (``config``, ``resume``,
``progress``, ``checkpoint``, ``done`` ...) so that a run's log can be grepped
or parsed back into dictionaries with :func:`parse_record`.
"""

from __future__ import annotations

import logging
import sys
import time
from pathlib import Path
from typing import Any, Optional

_LOGGER_NAME = "pygsquig_b200.run"


def _value(v: Any) -> str:
    if isinstance(v, float):
        return f"{v:.6g}"
    s = str(v)
    return f'"{s}"' if (" " in s or not s) else s


class _ElapsedFormatter(logging.Formatter):
    """Prefixes each record with the seconds since the log was opened."""

    def __init__(self, t0: float):
        super().__init__()
        self.t0 = t0

    def format(self, record: logging.LogRecord) -> str:
        return f"{record.created - self.t0:9.2f}s {record.levelname[0]} {record.getMessage()}"


class RunLog:
    """Structured run log.  ``event(name, **fields)`` writes one record."""

    def __init__(self, output_dir: Optional[Path] = None, level: str = "INFO"):
        self.t0 = time.time()
        self.logger = logging.getLogger(_LOGGER_NAME)
        self.logger.setLevel(logging.DEBUG)
        self.logger.propagate = False
        for h in list(self.logger.handlers):
            self.logger.removeHandler(h)
            h.close()
        fmt = _ElapsedFormatter(self.t0)
        out = logging.StreamHandler(sys.stdout)
        out.setLevel(getattr(logging, level.upper()))
        out.setFormatter(fmt)
        self.logger.addHandler(out)
        self.path = None
        if output_dir is not None:
            self.path = Path(output_dir) / "logs" / "run.log"
            self.path.parent.mkdir(parents=True, exist_ok=True)
            fh = logging.FileHandler(self.path)
            fh.setLevel(logging.DEBUG)
            fh.setFormatter(fmt)
            self.logger.addHandler(fh)

    # -- records -------------------------------------------------------------
    def event(self, name: str, level: int = logging.INFO, **fields) -> None:
        body = " ".join(f"{k}={_value(v)}" for k, v in fields.items())
        self.logger.log(level, f"{name} {body}".rstrip())

    def info(self, text: str, **fields) -> None:
        self.event("note", msg=text, **fields)

    def warning(self, text: str, **fields) -> None:
        self.event("warn", logging.WARNING, msg=text, **fields)

    # -- the driver's events ---------------------------------------------------
    def started(self, config, device: str) -> None:
        f = config.forcing
        self.event("start", N=config.grid.N, L=config.grid.L, alpha=config.solver.alpha,
                   nu_p=config.solver.dissipation.nu_p, t_end=config.simulation.t_end, device=device,
                   ring_kf=(f.kf if f else None), ring_eps=(f.epsilon if f else None))

    def progress(self, t: float, step: int, dt: float, diagnostics: dict, eta_seconds: Optional[float]) -> None:
        keep = {k: diagnostics[k] for k in ("energy", "enstrophy", "theta_rms", "cfl") if k in diagnostics}
        if eta_seconds is not None and eta_seconds > 0:
            keep["eta_s"] = int(eta_seconds)
        self.event("progress", t=t, step=step, dt=dt, **keep)

    def wrote(self, kind: str, path: Path, t: float, step: int) -> None:
        self.event(kind, logging.INFO if kind == "checkpoint" else logging.DEBUG, file=Path(path).name, t=t,
                   step=step)

    def finished(self, t: float, steps: int, wall_s: float) -> None:
        self.event("done", t=t, steps=steps, wall_s=wall_s, steps_per_s=steps / max(wall_s, 1e-12))


def parse_record(line: str) -> dict:
    """Inverse of one record's body: ``'progress t=1 step=2'`` ->
    ``{'event': 'progress', 't': '1', 'step': '2'}`` (values stay strings;
    quoted values keep their spaces).  The elapsed-time and level prefix of a
    formatted line is skipped."""
    parts = line.strip().split(" ")
    if len(parts) >= 2 and parts[0].endswith("s") and len(parts[1]) == 1:
        parts = parts[2:]
    while parts and parts[0] == "":
        parts = parts[1:]
    out = {"event": parts[0] if parts else ""}
    key, buf = None, []
    for tok in parts[1:]:
        if key is None:
            k, _, v = tok.partition("=")
            if v.startswith('"') and not (len(v) > 1 and v.endswith('"')):
                key, buf = k, [v[1:]]
                continue
            out[k] = v.strip('"')
        else:
            if tok.endswith('"'):
                buf.append(tok[:-1])
                out[key] = " ".join(buf)
                key = None
            else:
                buf.append(tok)
    return out
