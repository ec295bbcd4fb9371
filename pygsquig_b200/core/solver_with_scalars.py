"""gSQG solver with passive scalars (mirrors pygsquig/core/solver_with_scalars.py:57-236).

Each step advances theta first, then every scalar one RK4 step with the
velocity of the new theta frozen over the four stages
(solver_with_scalars.py:163-171, passive_scalar.py:212-232):
    d_t s = -dealias(u.grad s) - kappa k2 s + S.
Supported sources: none, or ``MeanGradientSource`` (S = -G.u).
"""

from __future__ import annotations

from typing import Callable, Optional

import numpy as np
import torch

from ..exceptions import ConfigurationError, PassiveScalarError
from ..scalars.source_terms import MeanGradientSource
from ..scalars.state import MultiScalarState
from .solver import State, gSQGSolver


class gSQGSolverWithScalars(gSQGSolver):
    def __init__(self, grid, alpha: float, nu_p: float = 0.0, p: int = 8,
                 passive_scalars: Optional[dict] = None, **kw):
        super().__init__(grid, alpha, nu_p, p, **kw)
        self.species = {}
        for name, cfg in (passive_scalars or {}).items():
            self._add(name, cfg.get("kappa", 0.0), cfg.get("source"))

    def _add(self, name, kappa, source):
        if kappa < 0:
            raise PassiveScalarError(f"kappa must be non-negative, got {kappa}")
        if source is not None and not isinstance(source, MeanGradientSource):
            raise NotImplementedError(
                "GPU scalar stages support source=None or MeanGradientSource; got " + type(source).__name__)
        if len(self.species) >= 4:
            raise ConfigurationError("at most 4 passive scalars per solver")
        self.species[name] = {"kappa": float(kappa), "source": source}

    def add_passive_scalar(self, name: str, kappa: float = 0.0, source=None) -> None:
        if name in self.species:
            raise ConfigurationError(f"Scalar '{name}' already exists")
        self._add(name, kappa, source)

    def _scalar_tuples(self):
        out = []
        for cfg in self.species.values():
            s = cfg["source"]
            out.append((cfg["kappa"], s is not None, float(s.gx) if s else 0.0, float(s.gy) if s else 0.0))
        return tuple(out)

    def initialize(self, theta0=None, seed: Optional[int] = None, scalar_init: Optional[dict] = None) -> dict:
        base = super().initialize(theta0, seed)
        if not self.species:
            return base
        pl = self.plan()
        N = self.grid.N
        scalar_init = scalar_init or {}
        scal = {}
        for name in self.species:
            f0 = scalar_init.get(name)
            f0 = np.zeros((N, N)) if f0 is None else f0
            scal[name] = pl.to_spectral(pl.check_real(f0, name))
        out = dict(base)
        out["scalar_state"] = MultiScalarState(scalars=scal, time=0.0, diagnostics={})
        return out

    def step(self, state: dict, dt: float, forcing: Optional[Callable] = None, damping: Optional[Callable] = None,
             **kwargs) -> dict:
        if "scalar_state" not in state or state["scalar_state"] is None:
            return super().step(state, dt, forcing, damping, **kwargs)
        ss = state["scalar_state"]
        base = {k: v for k, v in state.items() if k != "scalar_state"}
        new = super().step(base, dt, forcing, damping, **kwargs)
        if self.species:
            # the plan the theta step just used (its scalar buffers serve the
            # scalar stages; ring and damping do not enter them)
            pl = self.__dict__.get("_step_plan") or self.plan()
            names = list(self.species)
            s_in = [pl.check_spectrum(ss.scalars[n], n) for n in names]
            s_out = [torch.empty_like(t) for t in s_in]
            pl.scalars_step(new["theta_hat"], s_in, s_out, dt)
            ss = MultiScalarState(scalars=dict(zip(names, s_out)), time=ss.time + dt, diagnostics={})
        out = dict(new)
        out["scalar_state"] = ss
        return out

    def get_diagnostics(self, state: dict) -> dict:
        base = {k: v for k, v in state.items() if k != "scalar_state"}
        d = super().get_diagnostics(base)
        ss = state.get("scalar_state")
        if ss is not None:
            pl = self.aux_plan()
            L, N = self.grid.L, self.grid.N
            for name, sh in ss.scalars.items():
                sh = pl.check_spectrum(sh, name)
                phys = pl.to_physical(sh)
                mean = float(sh[0, 0].real.item()) / N**2
                d.update({
                    f"{name}_mean": mean,
                    f"{name}_variance": pl.scalar_variance(sh),
                    f"{name}_max": float(phys.max().item()),
                    f"{name}_min": float(phys.min().item()),
                    f"{name}_total": mean * L * L,
                    f"{name}_source_integrated": 0.0,
                    f"{name}_dissipation_integrated": 0.0,
                })
        return d
