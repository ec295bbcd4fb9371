"""Passive-scalar state containers (mirrors pygsquig/scalars/state.py:13-138)."""

from __future__ import annotations

from typing import NamedTuple, Optional


class PassiveScalarState(NamedTuple):
    scalar_hat: object
    time: float
    total_source: float = 0.0
    total_dissipation: float = 0.0

    def to_dict(self) -> dict:
        return {"scalar_hat": self.scalar_hat, "time": self.time, "total_source": self.total_source,
                "total_dissipation": self.total_dissipation}

    @classmethod
    def from_dict(cls, d: dict) -> "PassiveScalarState":
        return cls(scalar_hat=d["scalar_hat"], time=d.get("time", 0.0), total_source=d.get("total_source", 0.0),
                   total_dissipation=d.get("total_dissipation", 0.0))


class MultiScalarState(NamedTuple):
    scalars: dict
    time: float
    diagnostics: Optional[dict] = None

    def get_scalar(self, name: str):
        if name not in self.scalars:
            raise KeyError(f"Scalar '{name}' not found in state")
        return self.scalars[name]

    def update_scalar(self, name: str, scalar_hat) -> "MultiScalarState":
        s = dict(self.scalars)
        s[name] = scalar_hat
        return self._replace(scalars=s)
