"""Configuration and file formats of a run (mirrors pygsquig/io)."""

from .checkpoint import (
    load_checkpoint,
    load_diagnostics,
    load_output,
    save_checkpoint,
    save_diagnostics,
    save_output,
)
from .config import (
    DampingConfig,
    DissipationConfig,
    ForcingConfig,
    GridConfig,
    InitialConditionConfig,
    OutputConfig,
    PassiveScalarConfig,
    RunConfig,
    ScalarsConfig,
    ScalarSourceConfig,
    SimulationConfig,
    SolverConfig,
    TimeIntegrationConfig,
    load_config,
)

__all__ = [
    "RunConfig", "GridConfig", "SolverConfig", "ForcingConfig", "OutputConfig", "SimulationConfig",
    "InitialConditionConfig", "DissipationConfig", "DampingConfig", "TimeIntegrationConfig", "ScalarsConfig",
    "PassiveScalarConfig", "ScalarSourceConfig", "load_config", "save_checkpoint", "load_checkpoint",
    "save_output", "load_output", "save_diagnostics", "load_diagnostics",
]
