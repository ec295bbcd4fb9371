"""GPU parity of the kernel variants the large configurations run, and of the
passive-scalar passes with the mean-gradient source, against the float64
oracle (same seeded initial fields and host-drawn ring phases on both sides).

Variants covered here (launch shapes are chosen per N and precision):
  * FP64 radix-4 row pass at N = 512, 1024, 2048 (forced, damped IF-RK4);
  * FP32 radix-16 column pass (one or two column pairs per block), the
    radix-8 row pass and the last-stage row pass at N = 2048 and 4096;
  * the scalar row and column passes at N = 256 and 512 (FP64), 1024 and
    4096 (FP32; at 4096 the stage passes run at 64 registers with theta_{s+1}
    parked in shared memory), with and without a mean-gradient source;
  * the mean-gradient source S = -G.u (no reference counterpart: the oracle
    evaluates it as fft2(-(G_x u + G_y v)) from the velocity of the new theta,
    frozen over the scalar's RK stages as the reference freezes u, v,
    core/solver_with_scalars.py:131-178) at N = 64 and 256.

Tolerances (relative L2): FP64 <= 1e-11 per run of a few steps (a different
FFT factorisation, round-off only); FP32 < 2e-5 against the FP64 oracle
(single-precision transform round-off).  The longer runs print their error
and check looser bounds that allow for round-off growth in a chaotic flow.
"""

import functools
import os

import numpy as np
import pytest
import torch

from oracle import sqg_oracle as O

pytestmark = pytest.mark.gpu
TWO_PI = 2 * np.pi


@pytest.fixture(scope="module")
def P():
    from pygsquig_b200.build import build

    build()
    import pygsquig_b200 as P

    assert torch.cuda.is_available()
    O.set_fft_workers(len(os.sched_getaffinity(0)))  # threaded oracle FFTs at the large sizes
    yield P
    O.set_fft_workers(1)


def rel(a, b):
    a = a.detach().to(torch.complex128).cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def blob(N, cx, cy, w=0.3):
    x = np.arange(N) * TWO_PI / N
    X, Y = np.meshgrid(x, x, indexing="ij")
    dx = np.angle(np.exp(1j * (X - cx)))
    dy = np.angle(np.exp(1j * (Y - cy)))
    return np.exp(-(dx**2 + dy**2) / (2 * w**2))


def forced_case(N, alpha, seed, kf=None, spectrum="k4exp"):
    """Forced-dissipative IF-RK4 case scaled to N: ring at N/16 (at least 4),
    drag below kf/2, hyperviscosity with nu k_max^8 dt fixed."""
    kf = max(4.0, N / 16) if kf is None else kf
    go = O.make_grid(N, TWO_PI)
    if spectrum == "k4exp":
        th0 = O.random_phase_field(go, lambda k: k**4 * np.exp(-((k / max(N / 64, 2.0)) ** 2)), seed)
    else:
        th0 = O.random_phase_field(go, lambda k: k ** (-3.0), seed)
    nu = 1e-8 * (1024 / N) ** 8
    return go, th0, kf, nu


def run_pair(P, N, alpha, prec, n_steps, dt, seed, scalars=None, spectrum="k4exp"):
    """n_steps forced, damped IF-RK4 steps on the GPU and on the oracle.
    scalars: list of (kappa, G or None).  Returns (gpu state, oracle state)."""
    go, th0, kf, nu = forced_case(N, alpha, seed, spectrum=spectrum)
    rng = np.random.default_rng(seed + 1)
    phases = rng.uniform(0, TWO_PI, size=(n_steps, O.ring_mode_count(go, kf, 2.0)))
    ring_o, damp_o = O.RingForcing(kf, 2.0, 0.1), O.CombinedDamping(0.1, kf, nu, 8)
    g = P.make_grid(N, TWO_PI)
    ring, damp = P.RingForcing(kf, 2.0, 0.1), P.CombinedDamping(0.1, kf, nu, 8)
    if scalars:
        sp_o = {f"s{i}": {"kappa": k, "source": None if G is None else O.MeanGradientSource(*G)}
                for i, (k, G) in enumerate(scalars)}
        sp = {f"s{i}": {"kappa": k, "source": None if G is None else P.MeanGradientSource(*G)}
              for i, (k, G) in enumerate(scalars)}
        init = {f"s{i}": blob(N, 1.0 + 1.7 * i, 2.5 + 0.9 * i) for i in range(len(scalars))}
        so = O.gSQGSolverWithScalars(go, alpha, 0.0, 8, passive_scalars=sp_o, scheme="ifrk4")
        sto = so.initialize(theta0=th0, scalar_init=init)
        s = P.gSQGSolverWithScalars(g, alpha, 0.0, 8, passive_scalars=sp, precision=prec, scheme="ifrk4")
        st = s.initialize(theta0=th0, scalar_init=init)
    else:
        so = O.gSQGSolver(go, alpha, 0.0, 8, scheme="ifrk4")
        sto = so.initialize(theta0=th0)
        s = P.gSQGSolver(g, alpha, 0.0, 8, precision=prec, scheme="ifrk4")
        st = s.initialize(theta0=th0)
    for i in range(n_steps):
        sto = O.step_forced(so, sto, dt, ring_o, phases[i], damp_o)
        st = s.step(st, dt, forcing=ring.bind(phases[i], dt, g), damping=damp)
    torch.cuda.synchronize()
    return st, sto


def check_scalars(st, sto, tol, label):
    for name, ref in sto["scalars"].items():
        err = rel(st["scalar_state"].scalars[name], ref)
        print(f"{label} scalar {name}: rel L2 {err:.2e}")
        assert err < tol, (label, name, err)


@pytest.mark.parametrize("N,prec,tol", [(64, "float64", 1e-11), (64, "float32", 2e-5),
                                        (256, "float64", 1e-11), (256, "float32", 2e-5)])
def test_mean_gradient_source_vs_oracle(P, N, prec, tol):
    """Two mean-gradient scalars (G = (1, 0) and (0.3, -0.7)) and one without
    a source, advected by a forced gSQG flow (alpha = 0.5)."""
    scal = [(1e-4, (1.0, 0.0)), (1e-3, (0.3, -0.7)), (0.0, None)]
    st, sto = run_pair(P, N, 0.5, prec, 3, 2e-3 * 64 / N, 21 + N, scalars=scal)
    err = rel(st["theta_hat"], sto["theta_hat"])
    assert err < tol, err
    check_scalars(st, sto, tol, f"N={N} {prec}")


def test_mean_gradient_source_sign_and_normalisation(P):
    """theta = -U sin y with alpha = 1 gives psi = -U sin y, u = U cos y,
    v = 0, and no advection of theta or of a scalar that depends on y only.
    A zero scalar with kappa = 0 and G = (1, 0) then follows d_t s = -U cos y
    exactly: s(dt) = -U dt cos y.  G = (0, 1) leaves it at zero (v = 0)."""
    N, U, dt = 32, 0.3, 1e-2
    g = P.make_grid(N, TWO_PI)
    x = np.arange(N) * TWO_PI / N
    X, Y = np.meshgrid(x, x, indexing="ij")
    for G in ((1.0, 0.0), (0.0, 1.0)):
        s = P.gSQGSolverWithScalars(g, 1.0, 0.0, 8,
                                    passive_scalars={"c": {"kappa": 0.0, "source": P.MeanGradientSource(*G)}})
        st = s.initialize(theta0=-U * np.sin(Y), scalar_init={"c": np.zeros((N, N))})
        st = s.step(st, dt)
        sc = P.ifft2(st["scalar_state"].scalars["c"]).cpu().numpy()
        expect = -dt * G[0] * U * np.cos(Y)
        assert np.max(np.abs(sc - expect)) < 1e-15, (G, np.max(np.abs(sc - expect)))


@pytest.mark.parametrize("N", [512, 1024, 2048])
def test_fp64_radix4_row_pass_vs_oracle(P, N):
    """FP64 at the sizes whose row pass is radix 4 (N = 512 .. 2048)."""
    st, sto = run_pair(P, N, 1.0, "float64", 3, 2e-4, 40 + N)
    err = rel(st["theta_hat"], sto["theta_hat"])
    print(f"FP64 N={N} 3 forced IF-RK4 steps: rel L2 {err:.2e}")
    assert err <= 1e-11, err


@pytest.mark.parametrize("N,alpha", [(2048, 1.0), (4096, 0.5)])
def test_fp32_large_passes_vs_fp64_oracle(P, N, alpha):
    """FP32 radix-16 column pass, radix-8 row pass and the last-stage row
    pass (N = 2048: radix-4 row pass with the radix-16 column pass)."""
    st, sto = run_pair(P, N, alpha, "float32", 2, 5e-5, 60 + N, spectrum="kminus3")
    err = rel(st["theta_hat"], sto["theta_hat"])
    print(f"FP32 N={N} 2 forced IF-RK4 steps vs FP64 oracle: rel L2 {err:.2e}")
    assert err < 2e-5, err


@pytest.mark.parametrize("N,prec,tol", [(256, "float64", 1e-11), (512, "float64", 1e-11), (1024, "float32", 2e-5),
                                        (4096, "float32", 2e-5)])
def test_scalar_passes_vs_oracle(P, N, prec, tol):
    scal = [(1e-4, (1.0, 0.0)), (5e-4, None)]
    st, sto = run_pair(P, N, 1.0, prec, 2, 2e-4, 80 + N, scalars=scal)
    assert rel(st["theta_hat"], sto["theta_hat"]) < tol
    check_scalars(st, sto, tol, f"N={N} {prec}")


def test_config1_as_written_1000_steps(P):
    """Config 1 as written (N = 256, alpha = 1, nu = 1e-4, p = 8, dt = 1e-3,
    theta0 = sin 4x cos 4y + 1e-3 noise from seed 0, 1000 steps) with the
    integrating factor (explicit RK4 diverges at this nu): FP64 against the
    oracle's IF-RK4; energy and enstrophy compared too."""
    N, dt, nu, n = 256, 1e-3, 1e-4, 1000
    go = O.make_grid(N, TWO_PI)
    th0 = np.sin(4 * go.x) * np.cos(4 * go.y) + 1e-3 * np.random.default_rng(0).standard_normal((N, N))
    so = O.gSQGSolver(go, 1.0, nu, 8, scheme="ifrk4")
    sto = so.initialize(theta0=th0)
    for _ in range(n):
        sto = so.step(sto, dt)
    s = P.gSQGSolver(P.make_grid(N, TWO_PI), 1.0, nu, 8, scheme="ifrk4")
    st = s.multistep(s.initialize(theta0=th0), n, dt)
    err = rel(st["theta_hat"], sto["theta_hat"])
    from pygsquig_b200.utils.diagnostics import compute_enstrophy, compute_total_energy

    g = P.make_grid(N, TWO_PI)
    e_rel = abs(compute_total_energy(st["theta_hat"], g, 1.0) / O.compute_total_energy(sto["theta_hat"], go, 1.0) - 1)
    z_rel = abs(compute_enstrophy(st["theta_hat"], g, 1.0) / O.compute_enstrophy(sto["theta_hat"], go, 1.0) - 1)
    print(f"config 1 as written, {n} IF-RK4 steps FP64: theta_hat rel L2 {err:.2e}, energy {e_rel:.2e}, "
          f"enstrophy {z_rel:.2e}")
    assert err < 1e-10 and e_rel < 1e-10 and z_rel < 1e-10


@functools.lru_cache(maxsize=1)
def _config2_oracle(n):
    N, dt = 1024, 2e-4
    go = O.make_grid(N, TWO_PI)
    th0 = O.random_phase_field(go, lambda k: k**4 * np.exp(-((k / 10.0) ** 2)), 2)
    n_ring = O.ring_mode_count(go, 40.0, 2.0)
    phases = np.random.default_rng(1).uniform(0, TWO_PI, size=(n, n_ring))
    so = O.gSQGSolver(go, 1.0, 0.0, 8, scheme="ifrk4")
    ring_o, damp_o = O.RingForcing(40.0, 2.0, 0.1), O.CombinedDamping(0.1, 40.0, 1e-8, 8)
    sto = so.initialize(theta0=th0)
    for i in range(n):
        sto = O.step_forced(so, sto, dt, ring_o, phases[i], damp_o)
    return go, th0, phases, sto


@pytest.mark.parametrize("prec,tol", [("float64", 1e-10), ("float32", 1e-4)])
def test_config2_bounded_run(P, prec, tol):
    """Config 2 (N = 1024 forced-dissipative SQG: ring kf = 40, dk = 2,
    eps = 0.1; mu = 0.1, nu = 1e-8, p = 8 on CombinedDamping; dt = 2e-4;
    k^4 exp(-(k/10)^2) initial field, seed 2; phases from seed 1) over 50
    steps, FP64 and FP32 each against the FP64 oracle."""
    N, dt, n = 1024, 2e-4, 50
    go, th0, phases, sto = _config2_oracle(n)
    g = P.make_grid(N, TWO_PI)
    s = P.gSQGSolver(g, 1.0, 0.0, 8, precision=prec, scheme="ifrk4")
    st = s.multistep(s.initialize(theta0=th0), n, dt, forcing=P.RingForcing(40.0, 2.0, 0.1),
                     damping=P.CombinedDamping(0.1, 40.0, 1e-8, 8), noise=phases)
    err = rel(st["theta_hat"], sto["theta_hat"])
    from pygsquig_b200.utils.diagnostics import compute_total_energy

    e_rel = abs(compute_total_energy(st["theta_hat"], g, 1.0) / O.compute_total_energy(sto["theta_hat"], go, 1.0) - 1)
    print(f"config 2, {n} steps {prec} vs FP64 oracle: theta_hat rel L2 {err:.2e}, energy {e_rel:.2e}")
    assert err < tol and e_rel < tol


def test_config2_5000_steps_fp32_vs_fp64(P):
    """Config 2 over its 5000 steps: FP32 against FP64 on the GPU (the FP64
    path stands for the float64 oracle here -- test_config2_bounded_run pins
    it to the oracle over 50 steps; 5000 oracle steps at N = 1024 would take
    about half an hour of CPU).  Reports theta_hat, energy and enstrophy."""
    N, dt, n = 1024, 2e-4, 5000
    from pygsquig_b200.utils.diagnostics import compute_enstrophy, compute_total_energy
    from pygsquig_b200.utils.fields import random_phase_field

    g = P.make_grid(N, TWO_PI)
    th0 = random_phase_field(N, TWO_PI, lambda k: k**4 * np.exp(-((k / 10.0) ** 2)), 2)
    ring, damp = P.RingForcing(40.0, 2.0, 0.1), P.CombinedDamping(0.1, 40.0, 1e-8, 8)
    phases = np.random.default_rng(1).uniform(0, TWO_PI, size=(n, ring.n_modes(g)))
    out = {}
    for prec in ("float64", "float32"):
        s = P.gSQGSolver(g, 1.0, 0.0, 8, precision=prec, scheme="ifrk4")
        st = s.initialize(theta0=th0)
        for k in range(0, n, 500):
            st = s.multistep(st, 500, dt, forcing=ring, damping=damp, noise=phases[k:k + 500])
        torch.cuda.synchronize()
        out[prec] = (st["theta_hat"].to(torch.complex128), compute_total_energy(st["theta_hat"], g, 1.0),
                     compute_enstrophy(st["theta_hat"], g, 1.0))
    a, b = out["float32"], out["float64"]
    err = (torch.linalg.vector_norm(a[0] - b[0]) / torch.linalg.vector_norm(b[0])).item()
    e_rel, z_rel = abs(a[1] / b[1] - 1), abs(a[2] / b[2] - 1)
    print(f"config 2, {n} steps FP32 vs FP64: theta_hat rel L2 {err:.2e}, energy {e_rel:.2e}, enstrophy {z_rel:.2e}")
    assert np.isfinite(err) and err < 0.05 and e_rel < 0.01
