"""Scalar source terms supported by the GPU scalar stages."""

from __future__ import annotations

from dataclasses import dataclass


@dataclass
class MeanGradientSource:
    """S = -(gx u + gy v): a passive scalar s whose total field is
    s + gx x + gy y, advected by (u, v).

    No counterpart in the reference: its ``SourceTerm.__call__(scalar, grid,
    t)`` (scalars/source_terms.py:20-54) cannot see the velocity.  The source
    uses the velocity frozen over the scalar's RK4 stages, like the advection
    (solver_with_scalars.py:168-171).
    """

    gx: float = 1.0
    gy: float = 0.0
