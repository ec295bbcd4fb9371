"""Forcing and damping plug-ins of the hot path."""
from .damping import CombinedDamping, hyperviscosity, large_scale_damping
from .ring_forcing import BoundRingForcing, RingForcing

__all__ = ["RingForcing", "BoundRingForcing", "CombinedDamping", "large_scale_damping", "hyperviscosity"]
