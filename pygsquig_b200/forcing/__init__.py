"""Forcing and damping plug-ins of the hot path (mirrors pygsquig/forcing).

RingForcing and CombinedDamping run inside the stage kernels; the
deterministic and stochastic patterns are spectral terms that the solvers
add in the same stage update."""
from .damping import CombinedDamping, hyperviscosity, large_scale_damping
from .deterministic_forcing import (
    CheckerboardForcing,
    CombinedDeterministicForcing,
    DeterministicForcing,
    KolmogorovForcing,
    ShearLayerForcing,
    TaylorGreenForcing,
    TimeModulatedForcing,
    VortexPairForcing,
    make_kolmogorov_forcing,
    make_oscillating_forcing,
    make_taylor_green_forcing,
)
from .ring_forcing import BoundRingForcing, RingForcing
from .stochastic_forcing import (
    ColoredNoiseForcing,
    OrnsteinUhlenbeckForcing,
    StochasticForcing,
    StochasticVortexForcing,
    WhiteNoiseForcing,
    create_combined_stochastic_forcing,
)

__all__ = [
    "RingForcing", "BoundRingForcing", "CombinedDamping", "large_scale_damping", "hyperviscosity",
    "DeterministicForcing", "TaylorGreenForcing", "KolmogorovForcing", "CheckerboardForcing", "ShearLayerForcing",
    "VortexPairForcing", "TimeModulatedForcing", "CombinedDeterministicForcing", "make_taylor_green_forcing",
    "make_kolmogorov_forcing", "make_oscillating_forcing", "StochasticForcing", "WhiteNoiseForcing",
    "ColoredNoiseForcing", "StochasticVortexForcing", "OrnsteinUhlenbeckForcing",
    "create_combined_stochastic_forcing",
]
