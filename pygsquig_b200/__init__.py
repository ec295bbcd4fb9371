"""pygsquig_b200: B200-native RHS + RK4 hot path of pygSQuiG.

Drop-in for the reference's gSQGSolver / RingForcing / CombinedDamping /
passive-scalar path, running hand-written sm_100a CUDA kernels (libsqg.so)
through a ctypes C ABI.  No CPU fallback: the compute calls need the built
library and a CUDA device.
"""

__version__ = "0.1.0"

from .core.grid import Grid, fft2, ifft2, make_grid  # noqa: E402
from .core.solver import gSQGSolver  # noqa: E402
from .core.solver_with_scalars import gSQGSolverWithScalars  # noqa: E402
from .exceptions import (  # noqa: E402
    ConfigurationError,
    ForcingError,
    NumericalError,
    PassiveScalarError,
    SimulationError,
    pygSQuiGError,
)
from .forcing import CombinedDamping, RingForcing  # noqa: E402
from .scalars import MeanGradientSource, MultiScalarState  # noqa: E402

__all__ = [
    "Grid", "make_grid", "fft2", "ifft2", "gSQGSolver", "gSQGSolverWithScalars", "RingForcing",
    "CombinedDamping", "MeanGradientSource", "MultiScalarState", "pygSQuiGError", "ConfigurationError",
    "SimulationError", "NumericalError", "PassiveScalarError", "ForcingError",
]
