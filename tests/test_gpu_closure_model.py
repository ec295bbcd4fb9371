"""The learned closure as a solver term: the spectrum it adds against an
independent computation (numpy transforms + the float64 CNN oracle), and the
graph-replayed coarse step against the eager per-stage path."""

import math

import numpy as np
import pytest
import torch

from oracle import closure_oracle as CO

pytestmark = pytest.mark.gpu

TWO_PI = 2 * math.pi


def _field_hat(N, seed):
    rng = np.random.default_rng(seed)
    x = np.arange(N) * TWO_PI / N
    X, Y = np.meshgrid(x, x, indexing="ij")
    f = np.zeros((N, N))
    for _ in range(12):
        kx, ky = rng.integers(-20, 21, size=2)
        f += rng.standard_normal() * np.cos(kx * X + ky * Y + rng.uniform(0, TWO_PI))
    return np.fft.fft2(f)


def test_closure_term_matches_numpy_and_oracle():
    from pygsquig_b200.build import build

    build()
    from pygsquig_b200.closure.cnn import ClosureCNN
    from pygsquig_b200.closure.model import SubgridClosure

    N = 256
    net = ClosureCNN(N, N, max_batch=1, seed=5)
    sig_t, sig_p = 1.7, 3.0
    clo = SubgridClosure(net, N, TWO_PI, sig_t, sig_p)
    th_hat = _field_hat(N, 1)
    th = torch.as_tensor(th_hat, dtype=torch.complex64, device="cuda")
    term = clo(th).cpu().numpy().astype(np.complex128)
    y_phys = clo.physical(th).double().cpu().numpy()
    assert net.errors() == 0
    # independent: numpy inverse transform, float64 CNN, numpy forward transform, 2/3 disk
    theta = np.fft.ifft2(th_hat).real
    p = {k: v.detach().double().cpu().numpy() for k, v in net.p.items()}
    yo = CO.forward(p, theta[None] / sig_t)[0][0] * sig_p
    k1 = np.fft.fftfreq(N, 1.0 / N)
    kk = np.sqrt(k1[:, None] ** 2 + k1[None, :] ** 2)
    ref = np.fft.fft2(yo) * (kk < (2.0 / 3.0) * math.pi * N / TWO_PI)
    rel_phys = np.linalg.norm(y_phys - yo) / np.linalg.norm(yo)
    rel_spec = np.linalg.norm(term - ref) / np.linalg.norm(ref)
    assert rel_phys < 3e-2, rel_phys
    assert rel_spec < 3e-2, rel_spec
    assert np.abs(term[np.logical_not(kk < (2.0 / 3.0) * math.pi * N / TWO_PI)]).max() == 0.0


def test_graph_replayed_closure_step_matches_eager_steps():
    from pygsquig_b200 import CombinedDamping, RingForcing, gSQGSolver, make_grid
    from pygsquig_b200.closure.cnn import ClosureCNN
    from pygsquig_b200.closure.model import ClosureSolver, SubgridClosure

    N, dt, n = 256, 1e-3, 4
    g = make_grid(N, TWO_PI)
    s = gSQGSolver(g, 1.0, 0.0, 8, precision="float32", scheme="ifrk4")
    ring = RingForcing(20.0, 2.0, 0.1)
    damp = CombinedDamping(0.1, 20.0, 1e-22, 8)
    clo = SubgridClosure(ClosureCNN(N, N, max_batch=1, seed=2), N, TWO_PI, 2.0, 0.05)
    th0 = _field_hat(N, 3)
    noise = torch.as_tensor(np.random.default_rng(4).uniform(0, TWO_PI, (n, ring.n_modes(g))), device="cuda")
    st = s.initialize(theta0=np.fft.ifft2(th0).real)
    eager = st
    for i in range(n):
        eager = s.step(eager, dt, forcing=[ring.bind(noise[i], dt, g), clo], damping=damp)
    runner = ClosureSolver(s, clo, damp, ring)
    graph = runner.multistep(st, n, dt, noise)
    a = graph["theta_hat"].cpu().numpy().astype(np.complex128)
    b = eager["theta_hat"].cpu().numpy().astype(np.complex128)
    assert graph["step"] == n and abs(graph["time"] - n * dt) < 1e-15
    err = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert err < 1e-6, err
    # the closure changed the step (it is not a no-op)
    plain = s.multistep(st, n, dt, forcing=ring, damping=damp, noise=noise)
    c = plain["theta_hat"].cpu().numpy().astype(np.complex128)
    assert np.linalg.norm(a - c) / np.linalg.norm(c) > 1e-4
    assert clo.errors() == 0


def test_forcing_substeps_match_forcing_only_rk4():
    """sqg_ring_substeps against classic RK4 of d theta/dt = RingForcing(theta)
    (the oracle's restatement of ring_forcing.py:119-170), three sub-steps."""
    from oracle import sqg_oracle as O
    from pygsquig_b200 import RingForcing, gSQGSolver, make_grid

    N, dt = 64, 2e-3
    g = make_grid(N, TWO_PI)
    ring = RingForcing(8.0, 2.0, 0.1)
    s = gSQGSolver(g, 1.0, 0.0, 8, precision="float64")
    pl = s.plan(None, ring)
    rng = np.random.default_rng(5)
    th0 = _field_hat(N, 6) * 1e-2
    phases = rng.uniform(0, TWO_PI, (3, ring.n_modes(g)))
    th = torch.as_tensor(th0, dtype=torch.complex128, device="cuda").contiguous()
    pl.ring_substeps(th, 3, dt, torch.as_tensor(phases, device="cuda"))
    og = O.make_grid(N, TWO_PI)
    ro = O.RingForcing(8.0, 2.0, 0.1)
    ref = th0.copy()
    for m in range(3):
        ref = O.rk4_step(ref, lambda t: ro(t, phases[m], dt, og), dt)
    got = th.cpu().numpy()
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < 1e-12, err
    assert np.linalg.norm(got - th0) / np.linalg.norm(th0) > 1e-6  # the forcing acted


def test_free_running_errors_start_from_the_reference_spectrum():
    """The free-running evaluation's initial field carries the reference
    shell spectrum (shells 1..kf), and a short run stays finite with errors
    reported for every shell k <= kf."""
    from pygsquig_b200.build import build

    build()
    from pygsquig_b200.closure import experiment as X

    cfg = X.Config()
    kf = int(cfg.kf)
    E_ref = 1e-2 * np.arange(1, kf + 1, dtype=np.float64) ** -1.5
    # no time steps of averaging beyond one sample, no spin-up: the first sample is 10 steps in
    r = X.free_running_errors(cfg, None, E_ref, t_spin=0.0, t_avg=cfg.sample_dt, seed=3)
    assert r["finite"] and len(r["rel_err_E"]) == kf and r["samples"] == 1
    # 10 coarse steps (0.01 time units) barely move the resolved large scales
    assert max(r["rel_err_E"][:5]) < 0.05, r["rel_err_E"][:5]
