"""Batched ensembles of independent gSQG realisations on one GPU.

The reference runs ensembles as replicas under ``jax.pmap`` (pygsquig/core/
multi_gpu.py:118-205).  Here every member of a size class (same N) advances
in the same kernel launches: one launch per pass of an RK stage covers all
members of the class (alpha and the passive scalars vary per member), and a
whole step of the class is replayed from one CUDA graph.  Members of
different N form separate classes.

When every size class is one of N = 128, 256, 512 (the default ``unified``
mode), the classes advance together: one launch per pass of every RK stage
covers every member and every scalar of every class (eight launches per
step), with the scalars one step behind theta inside the same launches
(``sqg_ensemble_multistep``).  Other sizes step class by class.

Each member is a gSQG field with its own alpha and 0..4 passive scalars
(diffusivity kappa, no source), stepped like
``gSQGSolverWithScalars.step``: theta first, then the scalars with theta's
new velocity frozen over the stages (solver_with_scalars.py:131-178).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._plan import PlanKey, _stream_ptr, get_plan

TWO_PI = 2 * np.pi


SqgMember = _lib.SqgMember


@dataclass
class Member:
    """One realisation: N, alpha, initial theta (physical) and scalars."""

    N: int
    alpha: float
    theta0: np.ndarray
    scalars0: Sequence[np.ndarray] = field(default_factory=list)
    kappa: Sequence[float] = field(default_factory=list)


class _Batch:
    def __init__(self, N, L, members: List[Member], nu_p, p, precision, scheme, thetas, scalars):
        lib = _lib.load()
        d = _lib.SqgDesc()
        d.N, d.L, d.alpha, d.nu_p, d.p = N, L, 0.0, nu_p, p
        d.p_damp = 8
        d.precision = _lib.SQG_F64 if precision == "float64" else _lib.SQG_F32
        d.scheme = _lib.SQG_EXPLICIT_RK4 if scheme == "explicit" else _lib.SQG_IF_RK4
        arr = (SqgMember * len(members))()
        for i, m in enumerate(members):
            arr[i].theta = thetas[i].data_ptr()
            arr[i].alpha = float(m.alpha)
            arr[i].n_scalars = len(scalars[i])
            for q, t in enumerate(scalars[i]):
                arr[i].scalars[q] = t.data_ptr()
                arr[i].kappa[q] = float(m.kappa[q])
        h = C.c_void_p()
        _lib.check(lib.sqg_batch_create(C.byref(d), len(members), arr, C.byref(h)))
        self._h, self._lib = h, lib
        nb = C.c_size_t()
        _lib.check(lib.sqg_batch_workspace_bytes(h, C.byref(nb)))
        self.workspace = torch.empty(int(nb.value) + 256, dtype=torch.uint8, device="cuda")
        base = self.workspace.data_ptr()
        _lib.check(lib.sqg_batch_set_workspace(h, base + ((-base) % 256), int(nb.value), _stream_ptr()))

    def multistep(self, n, dt, use_graph=True):
        _lib.check(self._lib.sqg_batch_multistep(self._h, int(n), float(dt), 1 if use_graph else 0, _stream_ptr()))

    def launches(self):
        n = C.c_int64()
        _lib.check(self._lib.sqg_batch_last_launch_count(self._h, C.byref(n)))
        return int(n.value)

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._lib.sqg_batch_destroy(self._h)
                self._h = None
        except Exception:
            pass


UNIFIED_SIZES = (128, 256, 512)


class _Unified:
    """The size classes' batches advanced by one multi-size launch per pass."""

    def __init__(self, batches):
        lib = _lib.load()
        arr = (C.c_void_p * len(batches))(*[b._h.value for b in batches])
        h = C.c_void_p()
        _lib.check(lib.sqg_ensemble_create(arr, len(batches), C.byref(h)))
        self._h, self._lib, self._batches = h, lib, batches  # the batches outlive the ensemble

    def multistep(self, n, dt, use_graph=True):
        _lib.check(self._lib.sqg_ensemble_multistep(self._h, int(n), float(dt), 1 if use_graph else 0,
                                                    _stream_ptr()))

    def launches(self):
        n = C.c_int64()
        _lib.check(self._lib.sqg_ensemble_last_launch_count(self._h, C.byref(n)))
        return int(n.value)

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._lib.sqg_ensemble_destroy(self._h)
                self._h = None
        except Exception:
            pass


class EnsembleSolver:
    """Advances a list of members together (all states stay on the GPU)."""

    def __init__(self, members: Sequence[Member], nu_p: float = 0.0, p: int = 8, L: float = TWO_PI,
                 precision: str = "float32", scheme: str = "ifrk4", unified: bool = True):
        if p not in (2, 4, 8):
            raise ValueError(f"p must be 2, 4, or 8, got {p}")
        self.members = list(members)
        self.precision, self.scheme, self.L = precision, scheme, L
        cdt = torch.complex128 if precision == "float64" else torch.complex64
        self.theta: List[torch.Tensor] = []
        self.scalars: List[List[torch.Tensor]] = []
        for m in self.members:
            if not -2 <= m.alpha <= 2:
                raise ValueError(f"alpha must be in [-2, 2], got {m.alpha}")
            pl = get_plan(PlanKey(N=m.N, L=L, alpha=0.0, nu_p=0.0, p=8, precision=precision, role="aux"))
            self.theta.append(pl.to_spectral(pl.check_real(m.theta0)).to(cdt))
            self.scalars.append([pl.to_spectral(pl.check_real(s0)).to(cdt) for s0 in m.scalars0])
        self.classes: Dict[int, tuple] = {}
        for N in sorted({m.N for m in self.members}):
            idx = [i for i, m in enumerate(self.members) if m.N == N]
            b = _Batch(N, L, [self.members[i] for i in idx], nu_p, p, precision, scheme,
                       [self.theta[i] for i in idx], [self.scalars[i] for i in idx])
            self.classes[N] = (idx, b)
        self.unified = None
        if unified and set(self.classes) <= set(UNIFIED_SIZES):
            self.unified = _Unified([b for _, (_, b) in sorted(self.classes.items())])
        self.time = 0.0
        self.step_count = 0

    def multistep(self, n_steps: int, dt: float, use_graph: bool = True) -> None:
        if self.unified is not None:
            self.unified.multistep(n_steps, dt, use_graph)
        else:
            for _, (_, b) in self.classes.items():
                b.multistep(n_steps, dt, use_graph)
        self.time += n_steps * dt
        self.step_count += n_steps
        self._last_n = n_steps

    def launches_per_step(self) -> float:
        """Kernel launches per ensemble step in the last multistep call
        (class by class: the one input pass per size class at the start
        excluded; unified: every launch of the call, divided by its steps)."""
        n = getattr(self, "_last_n", 0)
        if not n:
            return 0.0
        if self.unified is not None:
            return self.unified.launches() / n
        return (sum(b.launches() for _, (_, b) in self.classes.items()) - len(self.classes)) / n

    def state(self, i: int) -> dict:
        return {"theta_hat": self.theta[i], "time": self.time, "step": self.step_count,
                "scalars": list(self.scalars[i])}
