"""gSQG solver (mirrors pygsquig/core/solver.py:61-245 and the ``multistep``
of pygsquig/core/solver_optimized.py:168-199).

Solves  d_t theta + u.grad(theta) = F - D,  u = grad_perp (-Lap)^(-alpha/2) theta
pseudo-spectrally on the GPU.  The state is the reference's dict
``{"theta_hat": (N, N) complex tensor, "time": float, "step": int}``.

Forcing / damping protocol (solver.py:150-214).  ``step`` accepts:

* ``damping``: ``CombinedDamping`` (run inside the fused stage kernels) or any
  callable ``damping(theta_hat, **kwargs)`` returning a spectrum;
* ``forcing``: ``RingForcing.bind(key, dt, grid)`` (fused), a ``RingForcing``
  together with ``key=`` phases in kwargs (fused), or any callable
  ``forcing(theta_hat, **kwargs)``; or a list of such terms (their sum, e.g.
  a bound ring forcing plus a learned subgrid closure).

Callables the kernels do not carry are evaluated by the host on every RK
stage input and added to that stage's right-hand side, exactly where the
reference adds them (solver.py:170-178).

Extensions (keyword-only): ``precision="float32"`` runs the FFTs, Jacobian and
RK4 stages in FP32 (float64 kept for the exponentials and reductions);
``scheme="ifrk4"`` integrates the diagonal terms exactly (needed for stiff
hyperviscosity where the reference's explicit RK4 diverges).
"""

from __future__ import annotations

from typing import Callable, Optional

import numpy as np
import torch

from .._plan import Plan, PlanKey, get_plan, plan_generation
from ..exceptions import NumericalError
from .. import _lib
from ..forcing.damping import CombinedDamping
from ..forcing.ring_forcing import BoundRingForcing, RingForcing

State = dict


class gSQGSolver:
    """Solver for the generalised SQG equations on one GPU."""

    def __init__(self, grid, alpha: float, nu_p: float = 0.0, p: int = 8, *, precision: str = "float64",
                 scheme: str = "explicit", check_finite: bool = False):
        self.grid = grid
        self.alpha = alpha
        self.nu_p = nu_p
        self.p = p
        if not -2 <= alpha <= 2:
            raise ValueError(f"alpha must be in [-2, 2], got {alpha}")
        if p not in [2, 4, 8]:
            raise ValueError(f"p must be 2, 4, or 8, got {p}")
        if precision not in ("float64", "float32"):
            raise ValueError(f"precision must be 'float64' or 'float32', got {precision!r}")
        if scheme not in ("explicit", "ifrk4"):
            raise ValueError(f"scheme must be 'explicit' or 'ifrk4', got {scheme!r}")
        self.precision = precision
        self.scheme = scheme
        self.check_finite = check_finite

    # ---- plans ----
    def _scalar_tuples(self):
        return ()

    def plan_key(self, damping: Optional[CombinedDamping] = None, ring: Optional[RingForcing] = None,
                 role: str = "step") -> PlanKey:
        g = self.grid
        return PlanKey(
            N=g.N, L=float(g.L), alpha=float(self.alpha), nu_p=float(self.nu_p), p=int(self.p),
            precision=self.precision, scheme=self.scheme,
            damping=None if damping is None else damping.plan_tuple(),
            ring=None if ring is None else ring.plan_tuple(),
            scalars=self._scalar_tuples(), role=role,
        )

    def _cached_plan(self, damping, ring, role) -> Plan:
        # The plan cache keyed by PlanKey costs a dataclass construction and
        # hash per call; this per-solver lookup on plain tuples is what a step
        # pays on the host.  The key holds every input of plan_key.
        k = (plan_generation(), role, self.alpha, self.nu_p, self.p, self.precision, self.scheme,
             self._scalar_tuples(), None if damping is None else damping.plan_tuple(),
             None if ring is None else ring.plan_tuple(),
             torch.cuda.current_device() if torch.cuda.is_available() else -1)
        cache = self.__dict__.setdefault("_plans", {})
        pl = cache.get(k)
        if pl is None:
            if len(cache) > 32:
                cache.clear()
            pl = cache[k] = get_plan(self.plan_key(damping, ring, role=role))
        return pl

    def plan(self, damping=None, ring=None) -> Plan:
        return self._cached_plan(damping, ring, "step")

    def aux_plan(self) -> Plan:
        """Plan for transforms, velocity, RHS and diagnostics: its own
        workspace, so a forcing callable may use them between RK stages."""
        return self._cached_plan(None, None, "aux")

    @property
    def cdtype(self):
        return torch.complex128 if self.precision == "float64" else torch.complex64

    # ---- reference API ----
    def initialize(self, theta0=None, seed: Optional[int] = None) -> State:
        """solver.py:96-124.  A seeded random field is drawn on the host with
        numpy.random.default_rng(seed) (the reference uses jax.random)."""
        pl = self.plan()
        N = self.grid.N
        if theta0 is not None:
            th = pl.to_spectral(pl.check_real(theta0, "theta0"))
        elif seed is not None:
            noise = np.random.default_rng(seed).standard_normal((N, N))
            th = pl.to_spectral(pl.check_real(noise))
            k_cutoff = N // 8
            mask = torch.sqrt(self.grid.k2) < k_cutoff * 2 * np.pi / self.grid.L
            th = th * mask.to(th.device)
        else:
            th = torch.zeros((N, N), dtype=self.cdtype, device=pl.device)
        return {"theta_hat": th, "time": 0.0, "step": 0}

    def compute_velocity(self, theta_hat):
        """operators.py:159-181 -> (u, v) in physical space."""
        pl = self.aux_plan()
        return pl.velocity(pl.check_spectrum(theta_hat))

    def compute_hyperviscosity(self, theta_hat):
        """-nu_p k2^(p/2) theta_hat (operators.py:185-207)."""
        pl = self.aux_plan()
        return pl.hyperviscosity(pl.check_spectrum(theta_hat))

    def compute_rhs(self, theta_hat, forcing: Optional[Callable] = None, damping: Optional[Callable] = None,
                    **kwargs):
        """solver.py:150-180."""
        pl = self.aux_plan()
        th = pl.check_spectrum(theta_hat)
        rhs = pl.rhs(th)
        if forcing is not None:
            rhs = rhs + forcing(theta_hat, **kwargs)
        if damping is not None:
            rhs = rhs + damping(theta_hat, **kwargs)
        return rhs

    def _classify(self, forcing, damping, kwargs):
        """Split forcing/damping into what the kernels carry and host callables."""
        ring, phases_key, generic = None, None, []
        damp = None
        if isinstance(damping, CombinedDamping):
            damp = damping
        elif damping is not None:
            generic.append(damping)
        terms = list(forcing) if isinstance(forcing, (list, tuple)) else ([] if forcing is None else [forcing])
        for f in terms:
            if isinstance(f, (BoundRingForcing, RingForcing)) and ring is not None:
                raise ValueError("at most one RingForcing per step")
            if isinstance(f, BoundRingForcing):
                ring, phases_key = f.ring, f.key
            elif isinstance(f, RingForcing):
                if "key" not in kwargs:
                    raise TypeError("RingForcing passed directly needs key=<phases> (or use ring.bind(key, dt, grid))")
                ring, phases_key = f, kwargs["key"]
            else:
                generic.append(f)
        return damp, ring, phases_key, generic

    def step(self, state: State, dt: float, forcing: Optional[Callable] = None, damping: Optional[Callable] = None,
             **kwargs) -> State:
        """One RK4 step (solver.py:182-214)."""
        damp, ring, phases_key, generic = self._classify(forcing, damping, kwargs)
        pl = self.plan(damp, ring)
        self._step_plan = pl  # the scalar stages of the same step run on this plan
        th = pl.check_spectrum(state["theta_hat"])
        phases = pl.phases_tensor(phases_key) if ring is not None else None
        out = torch.empty_like(th)
        if not generic:
            pl.step(th, out, dt, phases)
        else:
            stage_buf = pl.buffer(_lib.SQG_BUF_STAGE, th.dtype, th.shape)
            pl.stage_begin(th)
            for s in range(1, 5):
                th_s = th if s == 1 else stage_buf
                extra = None
                for c in generic:
                    term = pl.check_spectrum(c(th_s, **kwargs), "forcing/damping term")
                    extra = term if extra is None else extra + term
                pl.stage(s, th, out, dt, extra, phases)
        if self.check_finite and pl.check_status():
            raise NumericalError("non-finite values in theta_hat")
        return {"theta_hat": out, "time": state["time"] + dt, "step": state["step"] + 1}

    def multistep(self, state: State, n_steps: int, dt: float, forcing=None, damping=None, noise=None,
                  use_graph: bool = True, **kwargs) -> State:
        """n_steps RK4 steps in one call (solver_optimized.py:168-199).

        Forcing/damping as in ``step``; a RingForcing needs ``noise`` of shape
        (n_steps, n_ring) (one row of ring phases per step).  Without ring
        forcing the step is captured once in a CUDA graph and replayed.
        """
        terms = list(forcing) if isinstance(forcing, (list, tuple)) else ([] if forcing is None else [forcing])
        terms = [f.ring if isinstance(f, BoundRingForcing) else f for f in terms]
        damp, ring, _, generic = self._classify(terms, damping, dict(kwargs, key=None))
        if generic:
            gen_f = [f for f in terms if not isinstance(f, RingForcing)]
            for i in range(n_steps):
                f = list(gen_f)
                if ring is not None:
                    f.append(ring.bind(None if noise is None else noise[i], dt, self.grid))
                state = self.step(state, dt, forcing=f, damping=damping, **kwargs)
            return state
        pl = self.plan(damp, ring)
        th = pl.check_spectrum(state["theta_hat"]).clone()
        phases = pl.phases_tensor(noise, n_steps) if ring is not None else None
        pl.multistep(th, n_steps, dt, phases, use_graph)
        if self.check_finite and pl.check_status():
            raise NumericalError("non-finite values in theta_hat")
        return {"theta_hat": th, "time": state["time"] + n_steps * dt, "step": state["step"] + n_steps}

    def get_diagnostics(self, state: State) -> dict:
        """solver.py:216-245 (kinetic energy, 1/2<theta^2>, max|theta|)."""
        pl = self.aux_plan()
        d = pl.diagnostics(pl.check_spectrum(state["theta_hat"]))
        return {
            "kinetic_energy": float(d[2]),
            "enstrophy": float(d[3]),
            "max_theta": float(d[4]),
            "time": float(state["time"]),
            "step": int(state["step"]),
        }
