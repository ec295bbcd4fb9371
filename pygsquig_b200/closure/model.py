"""The learned subgrid closure as a forcing term of the coarse solve, and a
coarse solver that replays its step (closure included) as a CUDA graph.

The closure models the nonlinear term the coarse grid cannot carry,
    Pi = filter(-mask fft2(u.grad theta)) - (-mask_c fft2(u_c.grad theta_c)),
with theta_c = filter(theta) (the sharp filter of spectral.SpectralFilter).
It is evaluated on every RK stage input: theta_s -> physical theta (library
transform) -> CNN (library kernels, BF16 tensor cores) -> Pi(x, y).  As a
generic forcing term (``SubgridClosure.__call__``) Pi is transformed,
restricted to the coarse dealiased disk and added to that stage's
right-hand side, exactly where the solver adds any forcing term; the coarse
solver below instead hands Pi(x, y) to the stage kernels
(sqg_stage_physical), which subtract it from u.grad(theta) before the
forward transform and dealias the sum -- the same term without a separate
transform.
"""

from __future__ import annotations

import math
from typing import Optional

import numpy as np
import torch

from .. import _lib
from .._plan import PlanKey, get_plan
from ..exceptions import NumericalError
from ..forcing.damping import CombinedDamping
from ..forcing.ring_forcing import RingForcing
from .cnn import ClosureCNN
from .spectral import _kmag


class SubgridClosure:
    """forcing(theta_hat) -> closure spectrum (a term for gSQGSolver.step).

    ``sigma_theta`` / ``sigma_pi`` are the training normalisation: the CNN
    maps theta / sigma_theta to Pi / sigma_pi.
    """

    def __init__(self, net: ClosureCNN, N: int, L: float, sigma_theta: float, sigma_pi: float,
                 k_cut: Optional[float] = None, precision: str = "float32"):
        if net.H != N or net.W != N:
            raise ValueError("the network was built for another grid")
        self.net, self.N, self.L = net, N, L
        self.sigma_theta, self.sigma_pi = float(sigma_theta), float(sigma_pi)
        self.plan = get_plan(PlanKey(N=N, L=L, alpha=0.0, nu_p=0.0, p=8, precision=precision, role="closure"))
        dev = self.plan.device
        self.k_cut = (2.0 / 3.0) * math.pi * N / L if k_cut is None else k_cut
        self.mult = (_kmag(N, L, dev) < self.k_cut).to(self.plan.cdtype)
        self.phys = torch.empty((N, N), dtype=self.plan.rdtype, device=dev)
        self.x = torch.empty((1, N, N), dtype=torch.float32, device=dev)
        self.spec = torch.empty((N, N), dtype=self.plan.cdtype, device=dev)
        self.yspec_in = torch.empty((N, N), dtype=self.plan.rdtype, device=dev)

    def physical(self, theta_hat: torch.Tensor, normalised: bool = False) -> torch.Tensor:
        """CNN output Pi (FP32 [N, N]) for a coarse spectrum; the
        normalisation is folded into the first and last layers."""
        if self.plan.rdtype == torch.float32:
            self.plan.to_physical(theta_hat, out=self.x[0])
        else:
            self.plan.to_physical(theta_hat, out=self.phys)
            self.x[0].copy_(self.phys)
        return self.net.forward(self.x, in_scale=1.0 / self.sigma_theta,
                                out_scale=1.0 if normalised else self.sigma_pi)[0]

    def source(self, theta_hat: torch.Tensor) -> torch.Tensor:
        """Pi in physical space in the plan precision (the form the solver's
        stage kernels add to the advective term, sqg_stage_physical)."""
        y = self.physical(theta_hat)
        if self.yspec_in.dtype != y.dtype:
            self.yspec_in.copy_(y)
            return self.yspec_in
        return y

    def __call__(self, theta_hat: torch.Tensor, **kwargs) -> torch.Tensor:
        y = self.physical(theta_hat)
        if self.yspec_in.dtype != y.dtype:
            self.yspec_in.copy_(y)
            y = self.yspec_in
        self.plan.to_spectral(y, out=self.spec)
        return self.spec * self.mult

    def errors(self) -> int:
        return self.net.errors()

    # ---- persistence ----
    def save(self, path: str, **meta) -> None:
        d = {k: v.numpy() for k, v in self.net.state_dict().items()}
        np.savez(path, sigma_theta=self.sigma_theta, sigma_pi=self.sigma_pi, N=self.N, L=self.L, k_cut=self.k_cut,
                 meta=np.array(repr(meta)), **d)

    @classmethod
    def load(cls, path: str, max_batch: int = 1, precision: str = "float32") -> "SubgridClosure":
        z = np.load(path)
        N = int(z["N"])
        net = ClosureCNN(N, N, max_batch=max_batch)
        net.load_state_dict({k: torch.as_tensor(z[k]) for k, _ in ClosureCNN.SHAPES})
        return cls(net, N, float(z["L"]), float(z["sigma_theta"]), float(z["sigma_pi"]), float(z["k_cut"]),
                   precision)


class ClosureSolver:
    """Coarse gSQG solve with ring forcing / damping plus a learned closure on
    every RK stage; ``multistep`` captures one step (4 closure evaluations and
    4 fused stages) in a CUDA graph and replays it.

    ``forcing_substeps = m > 0`` splits the ring forcing off the RK stages:
    each step of length dt applies m forcing-only RK4 sub-steps of dt / m
    (half before the stages, half after; Strang splitting), each with its own
    phases (sqg_ring_substeps).  The reference's rescaled white-noise forcing
    injects an amount of energy that depends on the step it is integrated
    with (the rescale eps / <theta F> is singular where the overlap crosses
    zero), so a coarse solve whose step is m times the DNS step sees the DNS's
    forcing statistics only when the forcing keeps the DNS step.
    """

    def __init__(self, solver, closure: Optional[SubgridClosure], damping: Optional[CombinedDamping] = None,
                 ring: Optional[RingForcing] = None, forcing_substeps: int = 0):
        if solver.scheme != "ifrk4" and solver.scheme != "explicit":
            raise ValueError("unknown scheme")
        if forcing_substeps and ring is None:
            raise ValueError("forcing_substeps needs a RingForcing")
        self.solver, self.closure, self.damping, self.ring = solver, closure, damping, ring
        self.m = int(forcing_substeps)
        self.pl = solver.plan(damping, None if self.m else ring)
        self.pl_ring = solver.plan(damping, ring) if ring is not None else None
        N = solver.grid.N
        dev = self.pl.device
        self.n_ring = self.pl_ring.n_ring if self.pl_ring is not None else 0
        self.th_a = torch.zeros((N, N), dtype=self.pl.cdtype, device=dev)
        self.th_b = torch.zeros_like(self.th_a)
        self.ph = torch.zeros((max(self.m, 1), max(self.n_ring, 1)), dtype=torch.float64, device=dev)
        self.graph = None
        self.graph_dt = None

    @property
    def noise_rows_per_step(self) -> int:
        """Rows of ring phases one step consumes (m with split forcing, else 1)."""
        return max(self.m, 1)

    def _body(self, dt):
        pl = self.pl
        stage_buf = pl.buffer(_lib.SQG_BUF_STAGE, self.th_a.dtype, self.th_a.shape)
        ph = self.ph[0] if (self.ring is not None and not self.m) else None
        m1 = self.m // 2
        if self.m:
            self.pl_ring.ring_substeps(self.th_a, m1, dt / self.m, self.ph[:m1])
        pl.stage_begin(self.th_a)
        for s in range(1, 5):
            th_s = self.th_a if s == 1 else stage_buf
            if self.closure is not None:
                pl.stage_physical(s, self.th_a, self.th_b, dt, self.closure.source(th_s), ph)
            else:
                pl.stage(s, self.th_a, self.th_b, dt, None, ph)
        self.th_a.copy_(self.th_b)
        if self.m:
            self.pl_ring.ring_substeps(self.th_a, self.m - m1, dt / self.m, self.ph[m1:])

    def _capture(self, dt):
        cur = torch.cuda.current_stream()
        side = torch.cuda.Stream()
        side.wait_stream(cur)
        save = self.th_a.clone()
        with torch.cuda.stream(side):
            self._body(dt)  # warm-up outside the capture (kernel attributes, allocator)
        cur.wait_stream(side)
        self.th_a.copy_(save)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, capture_error_mode="thread_local"):
            self._body(dt)
        self.graph, self.graph_dt = g, dt

    def multistep(self, state: dict, n_steps: int, dt: float, noise: Optional[torch.Tensor] = None,
                  timer: Optional[list] = None) -> dict:
        """n_steps steps; ``noise``: device float64 ring phases, one row per
        step ([n_steps, n_ring]), or m rows per step with split forcing
        ([n_steps * m, n_ring]).  ``timer`` (a list) receives (start, end)
        CUDA events around the replays."""
        rows = self.noise_rows_per_step
        if self.ring is not None and (noise is None or noise.shape[0] < n_steps * rows):
            raise ValueError(f"ring forcing needs noise of shape ({n_steps * rows}, n_ring)")
        self.th_a.copy_(self.pl.check_spectrum(state["theta_hat"]))
        if self.graph is None or self.graph_dt != dt:
            self._capture(dt)
            self.th_a.copy_(self.pl.check_spectrum(state["theta_hat"]))
        ev = None
        if timer is not None:
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            ev[0].record()
        for i in range(n_steps):
            if self.ring is not None:
                self.ph.copy_(noise[i * rows:(i + 1) * rows])
            self.graph.replay()
        if ev is not None:
            ev[1].record()
            timer.append(ev)
        if self.solver.check_finite and self.pl.check_status():
            raise NumericalError("non-finite values in theta_hat")
        return {"theta_hat": self.th_a.clone(), "time": state["time"] + n_steps * dt,
                "step": state["step"] + n_steps}

    def tendency(self, theta_hat: torch.Tensor, aux_plan) -> torch.Tensor:
        """Resolved nonlinear tendency plus the closure term (for transfer
        spectra); ``aux_plan``: an inviscid plan of the coarse grid."""
        t = aux_plan.rhs(theta_hat)
        if self.closure is not None:
            t = t + self.closure(theta_hat)
        return t


def _main(argv=None) -> int:
    """Time the coarse closure solve: python -m pygsquig_b200.closure.model
    [--steps K] [--warmup W] [--no-closure] (graph replay, FP32 N = 256, the
    trained network when present, forcing split into DNS-sized sub-steps)."""
    import argparse
    import json
    import os

    from .experiment import Config, _solver

    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--no-closure", action="store_true")
    a = ap.parse_args(argv)
    from ..build import build

    build()
    cfg = Config()
    w = os.path.join(os.path.dirname(os.path.abspath(__file__)), "trained", "closure_weights.npz")
    clo = None
    if not a.no_closure:
        clo = (SubgridClosure.load(w) if os.path.exists(w)
               else SubgridClosure(ClosureCNN(cfg.N_c, cfg.N_c, max_batch=1), cfg.N_c, 2 * math.pi, 1.0, 1e-3))
    m = int(round(cfg.dt_c / cfg.dt))
    g, s, damp, ring = _solver(cfg, cfg.N_c, cfg.nu)
    runner = ClosureSolver(s, clo, damp, ring, forcing_substeps=m)
    rng = np.random.default_rng(0)
    st = s.initialize(theta0=rng.standard_normal((cfg.N_c, cfg.N_c)) * 0.3)
    noise = torch.as_tensor(rng.uniform(0, 2 * math.pi, ((a.warmup + a.steps) * m, runner.n_ring)), device="cuda")
    st = runner.multistep(st, a.warmup, cfg.dt_c, noise)
    tm = []
    st = runner.multistep(st, a.steps, cfg.dt_c, noise[a.warmup * m:], timer=tm)
    torch.cuda.synchronize()
    ms = sum(x.elapsed_time(y) for x, y in tm) / a.steps
    print(json.dumps({"ms_per_step": ms, "closure": clo is not None, "N": cfg.N_c, "dt": cfg.dt_c,
                      "forcing_substeps": m,
                      "finite": bool(torch.isfinite(torch.view_as_real(st["theta_hat"])).all())}))
    return 0


if __name__ == "__main__":
    raise SystemExit(_main())
