"""CPU float64 oracle for the pygSQuiG right-hand-side and RK4 hot path.

TEST INFRASTRUCTURE ONLY.  It checks the CUDA path: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` may
import it.  The product path (``pygsquig_b200``) never calls it and fails
loudly when its CUDA library is missing.

It restates, in NumPy float64, the algorithm of the reference JAX package
(dfielding14/pygSQuiG).  Every function cites the reference file:line it
follows.  Array layout matches the reference: ``ij`` indexing, row-major,
axis 0 = x / kx, axis 1 = y / ky; spectra are full (N, N) complex128.

Pinning.  The reference ships no golden vectors.  This restatement is pinned
(a) against the analytic known-answer tests of the reference's own test
suite (ported in ``tests/test_oracle_known_answers.py``) and (b) against
fixtures produced by importing the reference package itself in the build
container, through a NumPy-backed stand-in for the small part of the JAX API
it uses (``tests/golden/make_golden.py``).  The FFT library under (b) is
NumPy's pocketfft rather than XLA's, so (b) pins the algorithm to roundoff,
not XLA's last bits.

Randomness.  The reference draws noise with ``jax.random``; that stream is
not reproduced.  All random inputs (initial fields, ring-forcing phases) are
drawn on the host from ``numpy.random.default_rng(seed)`` and passed in.

Extensions that are not reference behaviour are labelled as such:
``scheme="ifrk4"`` (integrating-factor RK4, needed for the stiff hyperviscous
settings at which the explicit reference scheme diverges) and the
mean-gradient scalar source.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

try:  # multi-threaded FFT for the CPU baseline; plain NumPy otherwise
    import scipy.fft as _sfft
except Exception:  # pragma: no cover
    _sfft = None

_WORKERS = 1
_USE_SCIPY = False


def set_fft_workers(n: int) -> None:
    """Threads used by the oracle's FFTs.

    n == 1 (default): NumPy's FFT, the same arithmetic the fixtures were made
    with (bit-identical results).  n > 1: scipy.fft with ``workers=n`` (the
    threaded CPU baseline); results then differ at roundoff level.
    """
    global _WORKERS, _USE_SCIPY
    _WORKERS = max(1, int(n))
    _USE_SCIPY = _WORKERS > 1 and _sfft is not None


# ----------------------------------------------------------------------------
# Grid + FFT  (pygsquig/core/grid.py)
# ----------------------------------------------------------------------------


@dataclass
class Grid:
    """Restates ``Grid`` (pygsquig/core/grid.py:15-51)."""

    N: int
    L: float
    x: np.ndarray
    y: np.ndarray
    kx: np.ndarray
    ky: np.ndarray
    k2: np.ndarray
    dealias_mask: np.ndarray
    k1d: np.ndarray


def make_grid(N: int, L: float) -> Grid:
    """Restates ``make_grid`` (pygsquig/core/grid.py:72-107)."""
    if N % 2 != 0:  # grid.py:84-85
        raise ValueError(f"N must be even, got {N}")
    dx = L / N  # grid.py:88
    x1d = np.arange(N) * dx  # grid.py:89
    x, y = np.meshgrid(x1d, x1d, indexing="ij")  # grid.py:90
    k1d = np.fft.fftfreq(N, d=dx) * 2 * np.pi  # grid.py:94
    kx, ky = np.meshgrid(k1d, k1d, indexing="ij")  # grid.py:95
    k2 = kx**2 + ky**2  # grid.py:98
    k_max = np.pi * N / L  # grid.py:102
    dealias_cutoff = (2.0 / 3.0) * k_max  # grid.py:103
    dealias_mask = np.sqrt(k2) < dealias_cutoff  # grid.py:104-105
    return Grid(N, L, x, y, kx, ky, k2, dealias_mask, k1d)


def fft2(field: np.ndarray) -> np.ndarray:
    """Unnormalised forward 2-D FFT (pygsquig/core/grid.py:110-124)."""
    if _USE_SCIPY:
        return _sfft.fft2(field, workers=_WORKERS)
    return np.fft.fft2(field)


def ifft2(field_hat: np.ndarray) -> np.ndarray:
    """Inverse 2-D FFT with 1/N^2, real part (pygsquig/core/grid.py:127-138)."""
    if _USE_SCIPY:
        return _sfft.ifft2(field_hat, workers=_WORKERS).real
    return np.fft.ifft2(field_hat).real


# ----------------------------------------------------------------------------
# Spectral operators  (pygsquig/core/operators.py)
# ----------------------------------------------------------------------------


def gradient(theta_hat, grid):
    """operators.py:15-34."""
    return ifft2(1j * grid.kx * theta_hat), ifft2(1j * grid.ky * theta_hat)


def laplacian(theta_hat, grid):
    """operators.py:38-49."""
    return -grid.k2 * theta_hat


def fractional_laplacian(theta_hat, grid, alpha):
    """|k|^alpha with k=0 -> 0 (operators.py:53-72)."""
    k_mag = np.sqrt(grid.k2)
    k_safe = np.where(grid.k2 > 0, k_mag, 1.0)
    op = np.where(grid.k2 > 0, k_safe**alpha, 0.0)
    return op * theta_hat


def perpendicular_gradient(psi_hat, grid):
    """(u, v) = (-d_y psi, d_x psi) (operators.py:76-97)."""
    u = ifft2(-1j * grid.ky * psi_hat)
    v = ifft2(1j * grid.kx * psi_hat)
    return u, v


def jacobian(theta, u, v, grid):
    """u.grad(theta), dealiased on the output only (operators.py:101-130)."""
    theta_hat = fft2(theta)  # operators.py:117
    tx, ty = gradient(theta_hat, grid)  # :120
    jac = u * tx + v * ty  # :123
    jac_hat = fft2(jac) * grid.dealias_mask  # :126-127
    return ifft2(jac_hat)  # :130


def compute_streamfunction(theta_hat, grid, alpha):
    """psi_hat = |k|^-alpha theta_hat, k=0 -> 0 (operators.py:134-155)."""
    k_mag = np.sqrt(grid.k2)
    k_safe = np.where(grid.k2 > 0, k_mag, 1.0)
    inv = np.where(grid.k2 > 0, k_safe ** (-alpha), 0.0)
    return inv * theta_hat


def compute_velocity_from_theta(theta_hat, grid, alpha):
    """operators.py:159-181."""
    return perpendicular_gradient(compute_streamfunction(theta_hat, grid, alpha), grid)


def hyperviscosity(theta_hat, grid, nu_p, p):
    """-nu_p * k2**(p/2) * theta_hat with [0,0] = 0 (operators.py:185-207)."""
    d = -nu_p * (grid.k2 ** (p / 2)) * theta_hat
    d = np.array(d, dtype=np.complex128)
    d[0, 0] = 0.0
    return d


# ----------------------------------------------------------------------------
# Core RHS + solver  (pygsquig/core/solver.py)
# ----------------------------------------------------------------------------


def core_rhs(theta_hat, grid, alpha, nu_p, p, include_dissipation=True):
    """Restates ``_compute_core_rhs`` (pygsquig/core/solver.py:28-58)."""
    theta = ifft2(theta_hat)  # solver.py:46
    u, v = compute_velocity_from_theta(theta_hat, grid, alpha)  # :49
    advection = -jacobian(theta, u, v, grid)  # :52
    adv_hat = fft2(advection)  # :53
    if not include_dissipation:
        return adv_hat
    return adv_hat + hyperviscosity(theta_hat, grid, nu_p, p)  # :56-58


def large_scale_damping(theta_hat, grid, mu, kf):
    """-mu theta_hat for |k| < kf/2, k=0 included (forcing/damping.py:15-43)."""
    if mu == 0:
        return np.zeros_like(theta_hat)
    mask = np.sqrt(grid.k2) < kf / 2
    return -mu * theta_hat * mask


class CombinedDamping:
    """Restates ``CombinedDamping`` (pygsquig/forcing/damping.py:49-92)."""

    def __init__(self, mu=0.0, kf=20.0, nu_p=0.0, p=8):
        self.mu, self.kf, self.nu_p, self.p = mu, kf, nu_p, p
        if p not in [2, 4, 8]:  # damping.py:72-73
            raise ValueError(f"p must be 2, 4, or 8, got {p}")

    def __call__(self, theta_hat, grid):
        return large_scale_damping(theta_hat, grid, self.mu, self.kf) + hyperviscosity(
            theta_hat, grid, self.nu_p, self.p
        )


def rk4_step(state, rhs_fn, dt):
    """Classic RK4 (pygsquig/core/time_integrator.py:14-36)."""
    k1 = rhs_fn(state)
    k2 = rhs_fn(state + 0.5 * dt * k1)
    k3 = rhs_fn(state + 0.5 * dt * k2)
    k4 = rhs_fn(state + dt * k3)
    return state + dt * (k1 + 2 * k2 + 2 * k3 + k4) / 6


def ssp_rk3_step(state, rhs_fn, dt):
    """SSP-RK3 (pygsquig/core/time_integrator.py:39-67)."""
    k1 = rhs_fn(state)
    u1 = state + dt * k1
    k2 = rhs_fn(u1)
    u2 = (3 / 4) * state + (1 / 4) * u1 + (1 / 4) * dt * k2
    k3 = rhs_fn(u2)
    return (1 / 3) * state + (2 / 3) * u2 + (2 / 3) * dt * k3


def linear_operator(grid, nu_p, p, mu=0.0, kf_damp=0.0, nu_d=0.0, p_d=8):
    """Diagonal linear operator L(k) of the hyperviscous + drag terms.

    L = -nu_p k2^(p/2) [k != 0] - nu_d k2^(p_d/2) [k != 0] - mu [|k| < kf/2],
    i.e. the sum of ``hyperviscosity`` (operators.py:185-207) of the solver and
    of ``CombinedDamping`` plus ``large_scale_damping`` (damping.py:15-43).
    """
    L = -nu_p * grid.k2 ** (p / 2) - nu_d * grid.k2 ** (p_d / 2)
    L = np.array(L, dtype=np.float64)
    L[0, 0] = 0.0
    if mu != 0:
        L = L - mu * (np.sqrt(grid.k2) < kf_damp / 2)
    return L


def ifrk4_step(theta_hat, nonlin_fn, L, dt):
    """Integrating-factor RK4 (Lawson) -- EXTENSION, not reference behaviour.

    Solves d theta/dt = L theta + Nl(theta) with E = exp(L dt / 2):
      a = E (th + dt/2 k1);  b = E th + dt/2 k2;  c = E^2 th + dt E k3
      th' = E^2 th + dt/6 (E^2 k1 + 2 E (k2 + k3) + k4)
    """
    E = np.exp(L * (dt / 2))
    E2 = E * E
    k1 = nonlin_fn(theta_hat)
    k2 = nonlin_fn(E * (theta_hat + 0.5 * dt * k1))
    k3 = nonlin_fn(E * theta_hat + 0.5 * dt * k2)
    k4 = nonlin_fn(E2 * theta_hat + dt * E * k3)
    return E2 * theta_hat + dt / 6 * (E2 * k1 + 2 * E * (k2 + k3) + k4)


# ----------------------------------------------------------------------------
# Ring forcing  (pygsquig/forcing/ring_forcing.py)
# ----------------------------------------------------------------------------


def ensure_hermitian_symmetry(field_hat):
    """DC and Nyquist entries made real (ring_forcing.py:204-237)."""
    f = np.array(field_hat, dtype=np.complex128, copy=True)
    N = f.shape[0]
    f[0, 0] = f[0, 0].real
    if N % 2 == 0:
        N2 = N // 2
        f[N2, 0] = f[N2, 0].real
        f[0, N2] = f[0, N2].real
        f[N2, N2] = f[N2, N2].real
    return f


class RingForcing:
    """Restates ``RingForcing`` (pygsquig/forcing/ring_forcing.py:16-201).

    ``__call__(theta_hat, key, dt, grid)``: ``key`` is the host-drawn noise.
    It is either a full (N, N) array of phases in [0, 2pi) (what the
    reference's ``_generate_random_phases`` would return, ring_forcing.py:
    78-92) or a 1-D array of phases for the ring modes only, in row-major
    order of the ring mask.
    """

    def __init__(self, kf, dk=1.0, epsilon=0.1, tau_f=0.0, amplitude=None):
        self.kf, self.dk, self.epsilon, self.tau_f = kf, dk, epsilon, tau_f
        self.amplitude = math.sqrt(epsilon) if amplitude is None else amplitude  # :56-59
        self.forcing_state = None  # :62

    def get_forcing_mask(self, grid):
        """|sqrt(k2) - kf| <= dk/2 (ring_forcing.py:64-76)."""
        return np.abs(np.sqrt(grid.k2) - self.kf) <= self.dk / 2

    def phases_full(self, key, grid):
        key = np.asarray(key)
        if key.ndim == 2:
            return key
        mask = self.get_forcing_mask(grid)
        full = np.zeros((grid.N, grid.N))
        full[mask] = key
        return full

    def raw_forcing(self, key, dt, grid):
        """Forcing before the rate rescale (ring_forcing.py:134-150)."""
        mask = self.get_forcing_mask(grid)
        phases = np.exp(1j * self.phases_full(key, grid))  # :90-92
        forcing = self.amplitude * mask * phases  # :141
        if self.tau_f > 0:  # :144-145, OU update of :94-117
            if self.forcing_state is None:
                self.forcing_state = forcing
            else:
                decay = math.exp(-dt / self.tau_f)
                vf = math.sqrt(1 - decay**2)
                self.forcing_state = decay * self.forcing_state + vf * forcing
            forcing = self.forcing_state
        return ensure_hermitian_symmetry(forcing)  # :150

    def __call__(self, theta_hat, key, dt, grid):
        forcing = self.raw_forcing(key, dt, grid)
        theta = ifft2(theta_hat)  # :153
        force_phys = ifft2(forcing)  # :154
        rate = np.mean(theta * force_phys)  # :155
        scale = self.epsilon / rate if abs(rate) > 1e-10 else 1.0  # :161-165
        return scale * forcing  # :168

    def get_diagnostics(self, theta_hat, forcing, grid):
        """ring_forcing.py:172-201."""
        theta = ifft2(theta_hat)
        inj = np.mean(theta * ifft2(forcing))
        mask = self.get_forcing_mask(grid)
        return {
            "injection_rate": float(inj),
            "forcing_power": float(np.sum(np.abs(forcing * mask) ** 2)),
            "n_forced_modes": int(np.sum(mask)),
            "target_epsilon": self.epsilon,
        }


# ----------------------------------------------------------------------------
# Solver  (pygsquig/core/solver.py:61-245, solver_optimized.py:168-199)
# ----------------------------------------------------------------------------


class gSQGSolver:
    """Restates ``gSQGSolver`` (pygsquig/core/solver.py:61-245).

    ``scheme="explicit"`` is the reference's classic RK4 with hyperviscosity
    inside the RHS (time_integrator.py:14-36).  ``scheme="ifrk4"`` is the
    integrating-factor extension: the diagonal terms carried by the solver
    (``nu_p``) and by a ``CombinedDamping`` passed as ``damping`` are applied
    through exp(L dt/2); everything else is stepped as in RK4.
    """

    def __init__(self, grid, alpha, nu_p=0.0, p=8, scheme="explicit"):
        self.grid, self.alpha, self.nu_p, self.p = grid, alpha, nu_p, p
        if not -2 <= alpha <= 2:  # solver.py:91-92
            raise ValueError(f"alpha must be in [-2, 2], got {alpha}")
        if p not in [2, 4, 8]:  # solver.py:93-94
            raise ValueError(f"p must be 2, 4, or 8, got {p}")
        if scheme not in ("explicit", "ifrk4"):
            raise ValueError(f"unknown scheme {scheme!r}")
        self.scheme = scheme

    def initialize(self, theta0=None, seed=None):
        """solver.py:96-124 (random IC drawn from numpy default_rng)."""
        N = self.grid.N
        if theta0 is not None:
            theta_hat = fft2(np.asarray(theta0, dtype=np.float64))
        elif seed is not None:
            theta = np.random.default_rng(seed).standard_normal((N, N))
            theta_hat = fft2(theta)
            k_cutoff = N // 8
            mask = np.sqrt(self.grid.k2) < k_cutoff * 2 * np.pi / self.grid.L
            theta_hat = theta_hat * mask
        else:
            theta_hat = np.zeros((N, N), dtype=np.complex128)
        return {"theta_hat": theta_hat, "time": 0.0, "step": 0}

    def compute_velocity(self, theta_hat):
        return compute_velocity_from_theta(theta_hat, self.grid, self.alpha)

    def compute_hyperviscosity(self, theta_hat):
        return hyperviscosity(theta_hat, self.grid, self.nu_p, self.p)

    def compute_rhs(self, theta_hat, forcing=None, damping=None, **kwargs):
        """solver.py:150-180."""
        rhs = core_rhs(theta_hat, self.grid, self.alpha, self.nu_p, self.p)
        if forcing is not None:
            rhs = rhs + forcing(theta_hat, **kwargs)
        if damping is not None:
            rhs = rhs + damping(theta_hat, **kwargs)
        return rhs

    def _nonlinear(self, theta_hat, forcing, damping, kwargs):
        """RHS without the diagonal terms (used by the IF-RK4 extension)."""
        rhs = core_rhs(theta_hat, self.grid, self.alpha, 0.0, self.p, include_dissipation=False)
        if forcing is not None:
            rhs = rhs + forcing(theta_hat, **kwargs)
        if damping is not None and not isinstance(damping, CombinedDamping):
            rhs = rhs + damping(theta_hat, **kwargs)
        return rhs

    def linear_op(self, damping=None):
        if isinstance(damping, CombinedDamping):
            return linear_operator(
                self.grid, self.nu_p, self.p, damping.mu, damping.kf, damping.nu_p, damping.p
            )
        return linear_operator(self.grid, self.nu_p, self.p)

    def step(self, state, dt, forcing=None, damping=None, **kwargs):
        """solver.py:182-214."""
        th = state["theta_hat"]
        if self.scheme == "explicit":
            new = rk4_step(th, lambda t: self.compute_rhs(t, forcing, damping, **kwargs), dt)
        else:
            new = ifrk4_step(
                th,
                lambda t: self._nonlinear(t, forcing, damping, kwargs),
                self.linear_op(damping),
                dt,
            )
        return {"theta_hat": new, "time": state["time"] + dt, "step": state["step"] + 1}

    def multistep(self, state, n_steps, dt, forcing=None, damping=None, noise=None, **kwargs):
        """Loop of ``step``; ``lax.scan`` form in solver_optimized.py:168-199.

        ``forcing`` may be a RingForcing; then ``noise[i]`` is step i's phases.
        """
        for i in range(n_steps):
            if isinstance(forcing, RingForcing):
                key = noise[i]
                fr = forcing
                f = lambda th, _k=key, _f=fr: _f(th, _k, dt, self.grid)  # noqa: E731
            else:
                f = forcing
            d = damping
            if isinstance(damping, CombinedDamping):
                dm = damping
                d_call = lambda th, _d=dm: _d(th, self.grid)  # noqa: E731
                d = dm if self.scheme == "ifrk4" else d_call
            state = self.step(state, dt, forcing=f, damping=d, **kwargs)
        return state

    def get_diagnostics(self, state):
        """solver.py:216-245."""
        th = state["theta_hat"]
        theta = ifft2(th)
        u, v = self.compute_velocity(th)
        return {
            "kinetic_energy": float(0.5 * np.mean(u**2 + v**2)),
            "enstrophy": float(0.5 * np.mean(theta**2)),
            "max_theta": float(np.max(np.abs(theta))),
            "time": float(state["time"]),
            "step": int(state["step"]),
        }


def step_forced(solver, state, dt, ring, phases, damping):
    """One forced-dissipative step as the reference driver wires it.

    ``run.py:378-385`` and ``tests/test_integration.py:89-90,126``: the ring
    forcing is a lambda that captures (key, dt, grid) and CombinedDamping is
    called with ``grid=grid``.  The same phases are used at all 4 stages; the
    rescale factor is recomputed per stage from the stage theta.
    """
    grid = solver.grid
    f = None if ring is None else (lambda th: ring(th, phases, dt, grid))
    if solver.scheme == "explicit":
        d = None if damping is None else (lambda th: damping(th, grid))
        return solver.step(state, dt, forcing=f, damping=d)
    return solver.step(state, dt, forcing=f, damping=damping)


# ----------------------------------------------------------------------------
# Passive scalars  (pygsquig/scalars/passive_scalar.py, solver_with_scalars.py)
# ----------------------------------------------------------------------------


class MeanGradientSource:
    """NEW (no reference counterpart): S = -(G_x u + G_y v).

    Models theta_total = s + G.x advected by (u, v).  The reference's
    ``SourceTerm.__call__(scalar, grid, t)`` (scalars/source_terms.py:20-54)
    cannot see the velocity, so this source takes it explicitly.
    """

    def __init__(self, gx=1.0, gy=0.0):
        self.gx, self.gy = gx, gy

    def physical(self, u, v):
        return -(self.gx * u + self.gy * v)


def scalar_rhs(s_hat, u, v, grid, kappa, source_hat=None):
    """compute_passive_scalar_rhs (scalars/passive_scalar.py:24-103)."""
    s = ifft2(s_hat)  # :88
    adv_hat = fft2(-jacobian(s, u, v, grid))  # :41-42, :91
    rhs = adv_hat + (-kappa * grid.k2 * s_hat)  # :60, :94-97
    if source_hat is not None:  # :100-101
        rhs = rhs + source_hat
    return rhs


def scalar_step(s_hat, dt, u, v, grid, kappa, source=None, t=0.0, scheme="explicit"):
    """PassiveScalarEvolver.step (scalars/passive_scalar.py:212-232).

    u, v are frozen over the four stages; a source is evaluated at the stage
    scalar and at time t_n (``state.time``, :229).  ``source`` may be a
    callable(scalar_phys, grid, t) (reference SourceTerm protocol) or a
    MeanGradientSource (evaluated from u, v; constant over the step).
    """
    if isinstance(source, MeanGradientSource):
        src_hat = fft2(source.physical(u, v))
        src = lambda sh: src_hat  # noqa: E731
    elif source is not None:
        src = lambda sh: fft2(source(ifft2(sh), grid, t))  # noqa: E731  (:172-190)
    else:
        src = lambda sh: None  # noqa: E731
    if scheme == "explicit":
        return rk4_step(s_hat, lambda sh: scalar_rhs(sh, u, v, grid, kappa, src(sh)), dt)
    Ls = -kappa * grid.k2

    def nl(sh):
        r = fft2(-jacobian(ifft2(sh), u, v, grid))
        s_ = src(sh)
        return r if s_ is None else r + s_

    return ifrk4_step(s_hat, nl, Ls, dt)


class gSQGSolverWithScalars(gSQGSolver):
    """Restates ``gSQGSolverWithScalars`` (core/solver_with_scalars.py:57-236)."""

    def __init__(self, grid, alpha, nu_p=0.0, p=8, passive_scalars=None, scheme="explicit"):
        super().__init__(grid, alpha, nu_p, p, scheme)
        self.species = dict(passive_scalars or {})

    def initialize(self, theta0=None, seed=None, scalar_init=None):
        """solver_with_scalars.py:100-133; passive_scalar.py:320-339."""
        base = super().initialize(theta0, seed)
        if not self.species:
            return base
        scalar_init = scalar_init or {}
        N = self.grid.N
        scal = {}
        for name in self.species:
            f0 = scalar_init.get(name, np.zeros((N, N)))
            scal[name] = fft2(np.asarray(f0, dtype=np.float64))
        out = dict(base)
        out["scalars"] = scal
        return out

    def step(self, state, dt, forcing=None, damping=None, **kwargs):
        """solver_with_scalars.py:131-178: theta first, scalars with u,v at t_{n+1}."""
        base = {k: v for k, v in state.items() if k != "scalars"}
        new = super().step(base, dt, forcing, damping, **kwargs)
        if "scalars" not in state:
            return new
        u, v = self.compute_velocity(new["theta_hat"])  # :168
        out = dict(new)
        out["scalars"] = {}
        for name, cfg in self.species.items():
            out["scalars"][name] = scalar_step(
                state["scalars"][name],
                dt,
                u,
                v,
                self.grid,
                cfg.get("kappa", 0.0),
                cfg.get("source"),
                t=float(state["time"]),
                scheme=self.scheme,
            )
        return out


# ----------------------------------------------------------------------------
# Diagnostics  (pygsquig/utils/diagnostics.py, scalars/diagnostics.py)
# ----------------------------------------------------------------------------


def compute_total_energy(theta_hat, grid, alpha):
    """E = 1/2 sum k2^((alpha-2)/2) |th|^2 / N^2, [0,0]=0 (utils/diagnostics.py:171-190)."""
    k2s = np.where(grid.k2 > 0, grid.k2, 1.0)
    ed = 0.5 * k2s ** ((alpha - 2) / 2) * np.abs(theta_hat) ** 2
    ed[0, 0] = 0.0
    return float(np.sum(ed) / grid.N**2)


def compute_enstrophy(theta_hat, grid, alpha):
    """Z = 1/2 mean(|k|^alpha th|^2) * N^2 (utils/diagnostics.py:120-141)."""
    q = fractional_laplacian(theta_hat, grid, alpha)
    return float(0.5 * np.mean(np.abs(q) ** 2) * grid.N**2)


def compute_palinstrophy(theta_hat, grid, alpha):
    """utils/diagnostics.py:194-217."""
    k2s = np.where(grid.k2 > 0, grid.k2, 1.0)
    pd = 0.5 * k2s ** (1 + alpha) * np.abs(theta_hat) ** 2
    pd[0, 0] = 0.0
    return float(np.sum(pd) / grid.N**2)


def compute_energy_flux(theta_hat, forcing_hat, grid):
    """Re sum conj(th) F / N^2 (utils/diagnostics.py:145-167)."""
    if forcing_hat is None:
        return 0.0
    return float(np.real(np.sum(np.conj(theta_hat) * forcing_hat)) / grid.N**2)


def compute_energy_spectrum(theta_hat, grid, alpha):
    """Linear-bin shell spectrum (utils/diagnostics.py:22-84)."""
    k_mag = np.sqrt(grid.k2)
    k_safe = np.where(k_mag > 0, k_mag, 1.0)
    ed = 0.5 * k_safe ** (alpha - 2) * np.abs(theta_hat) ** 2
    ed[0, 0] = 0.0
    dk = 2 * np.pi / grid.L
    k_max = grid.N * dk / 2
    n_bins = min(grid.N // 4, 64)
    edges = np.linspace(0, k_max, n_bins + 1)
    centers = 0.5 * (edges[:-1] + edges[1:])
    E = np.zeros(n_bins)
    for i in range(n_bins):
        m = (k_mag >= edges[i]) & (k_mag < edges[i + 1])
        E[i] = np.sum(ed[m])
    E /= edges[1:] - edges[:-1]
    return centers, E


def compute_scalar_variance(s_hat):
    """<(s - <s>)^2> (scalars/diagnostics.py:156-168)."""
    s = ifft2(s_hat)
    sp = s - np.mean(s)
    return float(np.mean(sp**2))


# ----------------------------------------------------------------------------
# Seeded synthetic inputs of the benchmark configurations
# ----------------------------------------------------------------------------


def random_phase_field(grid, spectrum: Callable[[np.ndarray], np.ndarray], seed: int, rms=1.0):
    """Real field with random phases and |th(k)|^2 per shell ~ spectrum(|k|).

    Amplitude per mode = sqrt(spectrum(k) / (2 pi k)) (isotropic shell
    density), random phase from default_rng(seed); the real part of the
    inverse transform is taken and the field rescaled to the target rms.
    """
    rng = np.random.default_rng(seed)
    k = np.sqrt(grid.k2)
    ks = np.where(k > 0, k, 1.0)
    amp = np.sqrt(np.maximum(spectrum(ks), 0.0) / (2 * np.pi * ks))
    amp[0, 0] = 0.0
    ph = rng.uniform(0.0, 2 * np.pi, size=(grid.N, grid.N))
    th = np.fft.ifft2(amp * np.exp(1j * ph)).real
    s = np.sqrt(np.mean(th**2))
    if s > 0:
        th = th * (rms / s)
    return th


def ring_mode_count(grid, kf, dk):
    return int(np.sum(np.abs(np.sqrt(grid.k2) - kf) <= dk / 2))
