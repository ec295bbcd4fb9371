"""Passive scalars advected by the gSQG velocity."""
from .source_terms import MeanGradientSource
from .state import MultiScalarState, PassiveScalarState

__all__ = ["MeanGradientSource", "MultiScalarState", "PassiveScalarState"]
