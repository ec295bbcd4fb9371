"""Run configuration (mirrors pygsquig/io/config.py: same sections, field
names, defaults and validation messages, so the reference's YAML files load
unchanged)."""

from __future__ import annotations

import math
from dataclasses import asdict, dataclass, field
from pathlib import Path
from typing import Any, Optional, Union

import yaml


def _require(ok: bool, msg: str):
    if not ok:
        raise ValueError(msg)


@dataclass
class GridConfig:
    """config.py:15-33."""

    N: int = 256
    L: float = 2 * math.pi

    def __post_init__(self):
        _require(self.N > 0 and self.N % 2 == 0, f"N must be a positive even integer, got {self.N}")
        _require(self.L > 0, f"L must be positive, got {self.L}")


@dataclass
class DissipationConfig:
    """config.py:36-58."""

    type: str = "hyperviscosity"
    nu_p: float = 1.0e-16
    p: int = 8

    def __post_init__(self):
        _require(self.type in ("hyperviscosity", "viscosity"), f"Unknown dissipation type: {self.type}")
        _require(self.nu_p >= 0, f"nu_p must be non-negative, got {self.nu_p}")
        _require(self.p in (2, 4, 8), f"p must be 2, 4, or 8, got {self.p}")


@dataclass
class DampingConfig:
    """config.py:61-83."""

    type: str = "linear_drag"
    mu: float = 0.1
    k_cutoff_factor: float = 0.5

    def __post_init__(self):
        _require(self.type in ("linear_drag", "none"), f"Unknown damping type: {self.type}")
        _require(self.mu >= 0, f"mu must be non-negative, got {self.mu}")
        _require(self.k_cutoff_factor > 0, f"k_cutoff_factor must be positive, got {self.k_cutoff_factor}")


@dataclass
class TimeIntegrationConfig:
    """config.py:86-113."""

    method: str = "RK4"
    dt: float = 0.001
    adaptive_cfl: bool = True
    cfl_safety: float = 0.8
    dt_max: Optional[float] = None

    def __post_init__(self):
        _require(self.method in ("RK4", "SSP-RK3"), f"Unknown time integration method: {self.method}")
        _require(self.dt > 0, f"dt must be positive, got {self.dt}")
        _require(0 < self.cfl_safety < 1, f"cfl_safety must be in (0, 1), got {self.cfl_safety}")
        _require(self.dt_max is None or self.dt_max > 0, f"dt_max must be positive, got {self.dt_max}")


@dataclass
class SolverConfig:
    """config.py:116-134."""

    alpha: float
    dissipation: DissipationConfig = field(default_factory=DissipationConfig)
    damping: Optional[DampingConfig] = None
    time_integration: TimeIntegrationConfig = field(default_factory=TimeIntegrationConfig)

    def __post_init__(self):
        _require(-2 <= self.alpha <= 2, f"alpha must be in [-2, 2], got {self.alpha}")


@dataclass
class ForcingConfig:
    """config.py:137-168."""

    type: str = "ring"
    kf: float = 20.0
    dk: float = 1.0
    epsilon: float = 0.1
    tau_f: float = 0.0
    seed: Optional[int] = None

    def __post_init__(self):
        _require(self.type in ("ring", "none"), f"Unknown forcing type: {self.type}")
        _require(self.kf > 0, f"kf must be positive, got {self.kf}")
        _require(self.dk > 0, f"dk must be positive, got {self.dk}")
        _require(self.epsilon >= 0, f"epsilon must be non-negative, got {self.epsilon}")
        _require(self.tau_f >= 0, f"tau_f must be non-negative, got {self.tau_f}")


_FIELDS = {"theta", "vorticity", "streamfunction", "velocity", "scalars"}
_DIAGS = {"energy_spectrum", "scalar_flux", "enstrophy", "energy_flux"}


@dataclass
class OutputConfig:
    """config.py:171-197."""

    fields: list = field(default_factory=lambda: ["theta"])
    diagnostics: list = field(default_factory=lambda: ["energy_spectrum", "scalar_flux"])
    save_every_n_steps: Optional[int] = None
    compress: bool = True

    def __post_init__(self):
        bad = set(self.fields) - _FIELDS
        _require(not bad, f"Unknown fields: {bad}")
        bad = set(self.diagnostics) - _DIAGS
        _require(not bad, f"Unknown diagnostics: {bad}")


@dataclass
class SimulationConfig:
    """config.py:200-229."""

    t_end: float
    output_interval: float = 1.0
    checkpoint_interval: float = 10.0
    wall_time_limit: Optional[float] = None
    log_interval: float = 0.1

    def __post_init__(self):
        _require(self.t_end > 0, f"t_end must be positive, got {self.t_end}")
        for name in ("output_interval", "checkpoint_interval", "log_interval"):
            _require(getattr(self, name) > 0, f"{name} must be positive, got {getattr(self, name)}")
        _require(self.wall_time_limit is None or self.wall_time_limit > 0,
                 f"wall_time_limit must be positive, got {self.wall_time_limit}")


@dataclass
class ScalarSourceConfig:
    """config.py:232-245."""

    type: str
    parameters: dict = field(default_factory=dict)

    def __post_init__(self):
        _require(self.type in {"exponential", "localized", "chemical", "periodic", "none"},
                 f"Unknown source type: {self.type}")


@dataclass
class PassiveScalarConfig:
    """config.py:248-268."""

    name: str
    kappa: float = 0.0
    source: Optional[ScalarSourceConfig] = None
    initial_condition: str = "zero"
    initial_params: dict = field(default_factory=dict)

    def __post_init__(self):
        _require(self.kappa >= 0, f"kappa must be non-negative, got {self.kappa}")
        _require(self.initial_condition in {"zero", "random", "gaussian", "uniform"},
                 f"Unknown initial condition: {self.initial_condition}")


@dataclass
class ScalarsConfig:
    """config.py:271-285."""

    enabled: bool = False
    species: list = field(default_factory=list)

    def __post_init__(self):
        names = [s.name for s in self.species]
        _require(len(names) == len(set(names)), "Duplicate scalar names found")


@dataclass
class InitialConditionConfig:
    """config.py:288-308."""

    type: str = "random"
    checkpoint_path: Optional[str] = None
    amplitude: float = 1.0
    seed: Optional[int] = None

    def __post_init__(self):
        _require(self.type in ("random", "checkpoint", "function", "zero"),
                 f"Unknown initial condition type: {self.type}")
        _require(not (self.type == "checkpoint" and self.checkpoint_path is None),
                 "checkpoint_path required when type='checkpoint'")
        _require(self.amplitude > 0, f"amplitude must be positive, got {self.amplitude}")


def _drop_empty(d):
    """None values and empty dicts are left out of the serialised form
    (config.py:427-438)."""
    if isinstance(d, dict):
        return {k: _drop_empty(v) for k, v in d.items() if v is not None and (not isinstance(v, dict) or v)}
    return d


@dataclass
class RunConfig:
    """Top-level configuration (config.py:311-441)."""

    grid: GridConfig
    solver: SolverConfig
    forcing: Optional[ForcingConfig] = None
    scalars: Optional[ScalarsConfig] = None
    output: OutputConfig = field(default_factory=OutputConfig)
    simulation: SimulationConfig = field(default_factory=lambda: SimulationConfig(t_end=100.0))
    initial_condition: InitialConditionConfig = field(default_factory=InitialConditionConfig)

    @classmethod
    def from_yaml(cls, path: Union[str, Path]) -> "RunConfig":
        with open(path) as f:
            return cls.from_dict(yaml.safe_load(f))

    @classmethod
    def from_dict(cls, data: dict) -> "RunConfig":
        sd = dict(data.get("solver", {}))
        for key, typ in (("dissipation", DissipationConfig), ("damping", DampingConfig),
                         ("time_integration", TimeIntegrationConfig)):
            if key in sd and isinstance(sd[key], dict):
                sd[key] = typ(**sd[key])
        scalars = None
        sc = data.get("scalars")
        if sc and sc.get("enabled", False):
            species = []
            for sp in sc.get("species", []):
                src = sp.get("source")
                species.append(PassiveScalarConfig(
                    name=sp["name"], kappa=sp.get("kappa", 0.0),
                    source=None if src is None else ScalarSourceConfig(**src),
                    initial_condition=sp.get("initial_condition", "zero"),
                    initial_params=sp.get("initial_params", {})))
            scalars = ScalarsConfig(enabled=True, species=species)
        return cls(
            grid=GridConfig(**data.get("grid", {})),
            solver=SolverConfig(**sd),
            forcing=ForcingConfig(**data["forcing"]) if "forcing" in data else None,
            scalars=scalars,
            output=OutputConfig(**data.get("output", {})),
            simulation=SimulationConfig(**data.get("simulation", {"t_end": 100.0})),
            initial_condition=InitialConditionConfig(**data.get("initial_condition", {})),
        )

    def to_yaml(self, path: Union[str, Path]) -> None:
        with open(path, "w") as f:
            yaml.dump(self.to_dict(), f, default_flow_style=False, sort_keys=False)

    def to_dict(self) -> dict[Any, Any]:
        return dict(_drop_empty(asdict(self)))


def load_config(path: Union[str, Path]) -> RunConfig:
    """config.py:444-452."""
    return RunConfig.from_yaml(path)
