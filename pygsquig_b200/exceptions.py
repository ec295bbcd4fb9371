"""Exception hierarchy of pygSQuiG (mirrors pygsquig/exceptions.py:1-60)."""


class pygSQuiGError(Exception):
    """Base exception for all pygSQuiG errors."""


class ConfigurationError(pygSQuiGError):
    """Configuration parameters are invalid."""


class SimulationError(pygSQuiGError):
    """Raised during simulation execution."""


class NumericalError(SimulationError):
    """Numerical instability (non-finite values) was detected."""


class ValidationError(pygSQuiGError):
    """Parameter validation failed."""


class PassiveScalarError(pygSQuiGError):
    """Passive-scalar specific error."""


class SourceTermError(PassiveScalarError):
    """Source term computation failed."""


class ForcingError(pygSQuiGError):
    """Forcing configuration or computation failed."""
