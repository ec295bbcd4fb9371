"""GPU parity: the CUDA path against the reference's golden fixtures and the
float64 oracle.

Tolerances: the FP64 path must match to <= 1e-12 relative L2 per step on the
fixtures (roundoff of a different FFT factorisation) and <= 1e-11 after 100
RK4 steps at N=256 (the parity target).  FP32 results are compared with the
FP64 oracle at 2e-5 relative L2 (single-precision FFT roundoff).
"""

import os

import numpy as np
import pytest
import torch

from oracle import sqg_oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
TWO_PI = 2 * np.pi


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def cu(a, dtype=torch.complex128):
    return torch.as_tensor(np.asarray(a)).to("cuda", dtype)


@pytest.fixture(scope="module")
def P():
    from pygsquig_b200.build import build

    build()
    import pygsquig_b200 as P

    assert torch.cuda.is_available()
    return P


def test_roundtrip_and_parseval(P):
    for prec, tol in (("float64", 1e-14), ("float32", 3e-7)):
        g = P.make_grid(64, TWO_PI)
        rng = np.random.default_rng(0)
        f = rng.standard_normal((64, 64))
        dt = torch.float64 if prec == "float64" else torch.float32
        fh = P.fft2(torch.as_tensor(f, dtype=dt, device="cuda"))
        assert rel(fh, np.fft.fft2(f)) < tol * 10
        back = P.ifft2(fh)
        assert rel(back, f) < tol * 10
        # Parseval (test_grid.py:122-138)
        lhs = np.mean(f**2)
        rhs = float((fh.abs() ** 2).sum().item()) / 64**4
        assert abs(lhs - rhs) < 1e-12 * 10 if prec == "float64" else abs(lhs - rhs) < 1e-5


def test_rhs_matches_reference_fixtures(P):
    d = load("rhs")
    g = P.make_grid(32, TWO_PI)
    th = cu(d["theta_hat"])
    scale = np.linalg.norm(d["theta_hat"])
    for i in range(5):
        c = f"cases/case{i}/"
        s = P.gSQGSolver(g, float(d[c + "alpha"]), float(d[c + "nu_p"]), int(d[c + "p"]))
        r = s.compute_rhs(th).cpu().numpy()
        kmax = np.sqrt(2) * 16
        err = np.linalg.norm(r - d[c + "rhs"]) / (scale * max(1.0, kmax ** max(1 - float(d[c + "alpha"]), 0)))
        assert err < 1e-12, (i, err)
        u, v = s.compute_velocity(th)
        assert rel(u, d[c + "u"]) < 1e-12 and rel(v, d[c + "v"]) < 1e-12


def test_unforced_steps_match_fixtures(P):
    d = load("steps_unforced")
    g = P.make_grid(32, TWO_PI)
    s = P.gSQGSolver(g, float(d["alpha"]), float(d["nu_p"]), int(d["p"]))
    st = s.initialize(theta0=d["theta0"])
    assert rel(st["theta_hat"], d["traj"][0]) < 1e-14
    for i in range(1, d["traj"].shape[0]):
        st = s.step(st, float(d["dt"]))
        assert rel(st["theta_hat"], d["traj"][i]) < 1e-12, i
        dg = s.get_diagnostics(st)
        assert abs(dg["kinetic_energy"] - d["diag_ke"][i]) < 1e-12 * d["diag_ke"][i]
        assert abs(dg["enstrophy"] - d["diag_ens"][i]) < 1e-12 * d["diag_ens"][i]
        assert abs(dg["max_theta"] - d["diag_max"][i]) < 1e-12 * d["diag_max"][i]
    assert st["step"] == 10 and abs(st["time"] - 10 * float(d["dt"])) < 1e-15


def test_alpha05_steps_match_fixtures(P):
    d = load("steps_alpha05")
    g = P.make_grid(32, TWO_PI)
    s = P.gSQGSolver(g, float(d["alpha"]), float(d["nu_p"]), int(d["p"]))
    st = s.initialize(theta0=d["theta0"])
    for i in range(1, d["traj"].shape[0]):
        st = s.step(st, float(d["dt"]))
        assert rel(st["theta_hat"], d["traj"][i]) < 1e-12, i


@pytest.mark.parametrize("use_graph", [False, True])
def test_multistep_matches_fixture(P, use_graph):
    d = load("multistep")
    g = P.make_grid(32, TWO_PI)
    s = P.gSQGSolver(g, float(d["alpha"]), float(d["nu_p"]), int(d["p"]))
    st0 = s.initialize(theta0=d["theta0"])
    st = s.multistep(st0, int(d["n"]), float(d["dt"]), use_graph=use_graph)
    assert rel(st["theta_hat"], d["theta_hat"]) < 1e-12
    # multistep == repeated step, bit for bit
    st2 = st0
    for _ in range(int(d["n"])):
        st2 = s.step(st2, float(d["dt"]))
    assert torch.equal(st["theta_hat"], st2["theta_hat"])


@pytest.mark.parametrize("name", ["forced", "forced_dup_nu", "forced_ou"])
@pytest.mark.parametrize("path", ["fused", "generic"])
def test_forced_steps_match_fixtures(P, name, path):
    d = load(name)
    g = P.make_grid(32, TWO_PI)
    ring = P.RingForcing(float(d["kf"]), float(d["dk"]), float(d["eps"]), float(d["tau_f"]))
    damp = P.CombinedDamping(float(d["mu"]), float(d["kf_damp"]), float(d["nu_damp"]), int(d["p"]))
    s = P.gSQGSolver(g, 1.0, float(d["nu_solver"]), int(d["p"]))
    st = s.initialize(theta0=d["theta0"])
    dt = float(d["dt"])
    for i in range(d["phases"].shape[0]):
        if path == "fused":
            st = s.step(st, dt, forcing=ring.bind(d["phases"][i], dt, g), damping=damp)
        else:
            ph = d["phases"][i]
            st = s.step(st, dt, forcing=lambda th, _p=ph, **kw: ring(th, _p, dt, g), damping=damp, grid=g)
        assert rel(st["theta_hat"], d["traj"][i + 1]) < 1e-12, (i, rel(st["theta_hat"], d["traj"][i + 1]))


def test_generic_damping_callable(P):
    # test_solver.py:307-349: arbitrary callables through **kwargs
    g = P.make_grid(64, TWO_PI)
    s = P.gSQGSolver(g, 1.0, 0.0)
    so = O.gSQGSolver(O.make_grid(64, TWO_PI), 1.0, 0.0)
    th0 = np.sin(g.x.cpu().numpy())
    st, sto = s.initialize(theta0=th0), so.initialize(theta0=th0)
    damp = lambda th, **kw: -0.1 * th  # noqa: E731
    for _ in range(10):
        st = s.step(st, 0.1, damping=damp)
        sto = so.step(sto, 0.1, damping=damp)
    assert rel(st["theta_hat"], sto["theta_hat"]) < 1e-12

    def forcing(th, **kw):
        f = torch.zeros_like(th)
        f[1, 0] = 0.1
        f[0, 1] = 0.1
        return f

    def forcing_np(th, **kw):
        f = np.zeros_like(th)
        f[1, 0] = 0.1
        f[0, 1] = 0.1
        return f

    st = s.step(s.initialize(), 0.01, forcing=forcing)
    sto = so.step(so.initialize(), 0.01, forcing=forcing_np)
    assert rel(st["theta_hat"], sto["theta_hat"]) < 1e-12


def test_scalars_match_fixtures(P):
    d = load("scalars")
    g = P.make_grid(32, TWO_PI)
    s = P.gSQGSolverWithScalars(g, float(d["alpha"]), float(d["nu_p"]), int(d["p"]),
                                passive_scalars={"a": {"kappa": float(d["kappa_a"])},
                                                 "b": {"kappa": float(d["kappa_b"])}})
    st = s.initialize(theta0=d["theta0"], scalar_init={"a": d["a0"], "b": d["b0"]})
    for i in range(1, d["traj_a"].shape[0]):
        st = s.step(st, float(d["dt"]))
        assert rel(st["theta_hat"], d["traj_theta"][i]) < 1e-12
        assert rel(st["scalar_state"].scalars["a"], d["traj_a"][i]) < 1e-12, i
        assert rel(st["scalar_state"].scalars["b"], d["traj_b"][i]) < 1e-12, i
        dg = s.get_diagnostics(st)
        assert abs(dg["a_variance"] - d["var_a"][i]) < 1e-12 * d["var_a"][i]


def test_diagnostics_match_fixtures(P):
    from pygsquig_b200.utils import diagnostics as D

    d = load("diagnostics")
    g = P.make_grid(32, TWO_PI)
    th = cu(d["theta_hat"])
    for alpha in (1.0, 0.5, 0.0, 1.5):
        c = f"alphas/a{alpha}/"
        assert abs(D.compute_total_energy(th, g, alpha) - d[c + "energy"]) < 1e-12 * abs(d[c + "energy"])
        assert abs(D.compute_enstrophy(th, g, alpha) - d[c + "enstrophy"]) < 1e-12 * abs(d[c + "enstrophy"])
        assert abs(D.compute_palinstrophy(th, g, alpha) - d[c + "palinstrophy"]) < 1e-12 * abs(d[c + "palinstrophy"])
        kb, E = D.compute_energy_spectrum(th, g, alpha)
        assert np.allclose(kb, d[c + "k_bins"], rtol=1e-15)
        assert np.allclose(E, d[c + "E_k"], rtol=1e-12, atol=1e-300)


def test_parity_100_steps_N256(P):
    """Config-1 geometry (N=256, alpha=1, p=8, dt=1e-3, seeded IC) at the
    stable nu = 1e-16: <= 1e-11 relative L2 on theta_hat after 100 steps."""
    N, dt, nu = 256, 1e-3, 1e-16
    go = O.make_grid(N, TWO_PI)
    th0 = np.sin(4 * go.x) * np.cos(4 * go.y) + 1e-3 * np.random.default_rng(0).standard_normal((N, N))
    so = O.gSQGSolver(go, 1.0, nu, 8)
    sto = so.initialize(theta0=th0)
    g = P.make_grid(N, TWO_PI)
    s = P.gSQGSolver(g, 1.0, nu, 8)
    st = s.initialize(theta0=th0)
    for _ in range(100):
        sto = so.step(sto, dt)
    st = s.multistep(st, 100, dt)
    err = rel(st["theta_hat"], sto["theta_hat"])
    print("N=256 100-step FP64 rel L2 vs oracle:", err)
    assert err <= 1e-11
    e_gpu = s.get_diagnostics(st)
    e_ora = so.get_diagnostics(sto)
    assert abs(e_gpu["kinetic_energy"] - e_ora["kinetic_energy"]) < 1e-11 * e_ora["kinetic_energy"]


def test_ifrk4_matches_oracle_stiff(P):
    """Config-1 parameters as written (nu=1e-4, p=8: explicit RK4 diverges)
    at N=64 with the integrating-factor scheme, FP64 vs oracle."""
    N, dt, nu = 64, 1e-3, 1e-4
    go = O.make_grid(N, TWO_PI)
    th0 = np.sin(4 * go.x) * np.cos(4 * go.y) + 1e-3 * np.random.default_rng(0).standard_normal((N, N))
    so = O.gSQGSolver(go, 1.0, nu, 8, scheme="ifrk4")
    s = P.gSQGSolver(P.make_grid(N, TWO_PI), 1.0, nu, 8, scheme="ifrk4")
    sto, st = so.initialize(theta0=th0), s.initialize(theta0=th0)
    for _ in range(20):
        sto = so.step(sto, dt)
    st = s.multistep(st, 20, dt)
    assert rel(st["theta_hat"], sto["theta_hat"]) < 1e-11


def test_ifrk4_forced_damped_vs_oracle(P):
    N, dt = 64, 2e-3
    go = O.make_grid(N, TWO_PI)
    rng = np.random.default_rng(7)
    th0 = O.random_phase_field(go, lambda k: k**4 * np.exp(-((k / 5) ** 2)), 2)
    ring_o = O.RingForcing(10.0, 2.0, 0.1)
    damp_o = O.CombinedDamping(0.1, 10.0, 1e-8, 8)
    so = O.gSQGSolver(go, 1.0, 0.0, 8, scheme="ifrk4")
    n_ring = O.ring_mode_count(go, 10.0, 2.0)
    phases = rng.uniform(0, 2 * np.pi, size=(8, n_ring))
    sto = so.initialize(theta0=th0)
    for i in range(8):
        sto = O.step_forced(so, sto, dt, ring_o, phases[i], damp_o)
    s = P.gSQGSolver(P.make_grid(N, TWO_PI), 1.0, 0.0, 8, scheme="ifrk4")
    st = s.multistep(s.initialize(theta0=th0), 8, dt, forcing=P.RingForcing(10.0, 2.0, 0.1),
                     damping=P.CombinedDamping(0.1, 10.0, 1e-8, 8), noise=phases)
    assert rel(st["theta_hat"], sto["theta_hat"]) < 1e-11


def test_fp32_error_vs_fp64_oracle(P):
    N, dt = 128, 2e-3
    go = O.make_grid(N, TWO_PI)
    th0 = O.random_phase_field(go, lambda k: k**4 * np.exp(-((k / 10) ** 2)), 2)
    so = O.gSQGSolver(go, 1.0, 1e-16, 8)
    sto = so.initialize(theta0=th0)
    for _ in range(10):
        sto = so.step(sto, dt)
    s = P.gSQGSolver(P.make_grid(N, TWO_PI), 1.0, 1e-16, 8, precision="float32")
    st = s.multistep(s.initialize(theta0=th0), 10, dt)
    assert st["theta_hat"].dtype == torch.complex64
    err = rel(st["theta_hat"].to(torch.complex128), sto["theta_hat"])
    print("FP32 vs FP64 oracle, N=128, 10 steps:", err)
    assert err < 2e-5


@pytest.mark.parametrize("N", [128, 256, 512, 1024])
def test_fp32_forced_ifrk4_vs_fp64_oracle(P, N):
    """FP32 forced, damped IF-RK4 (the sizes whose row pass is radix 4, incl.
    the radix-2 first pass at N = 128 and 512) against the float64 oracle
    restatement: relative L2 < 2e-5 after 4 steps (FP32 transform round-off)."""
    dt, kf = 2e-4, N / 16
    go = O.make_grid(N, TWO_PI)
    rng = np.random.default_rng(N)
    th0 = O.random_phase_field(go, lambda k: k**4 * np.exp(-((k / (N / 64)) ** 2)), 3)
    ring_o = O.RingForcing(kf, 2.0, 0.1)
    damp_o = O.CombinedDamping(0.1, kf, 1e-8 * (1024 / N) ** 8, 8)
    so = O.gSQGSolver(go, 1.0, 0.0, 8, scheme="ifrk4")
    phases = rng.uniform(0, 2 * np.pi, size=(4, O.ring_mode_count(go, kf, 2.0)))
    sto = so.initialize(theta0=th0)
    for i in range(4):
        sto = O.step_forced(so, sto, dt, ring_o, phases[i], damp_o)
    s = P.gSQGSolver(P.make_grid(N, TWO_PI), 1.0, 0.0, 8, precision="float32", scheme="ifrk4")
    st = s.multistep(s.initialize(theta0=th0), 4, dt, forcing=P.RingForcing(kf, 2.0, 0.1),
                     damping=P.CombinedDamping(0.1, kf, 1e-8 * (1024 / N) ** 8, 8), noise=phases)
    err = rel(st["theta_hat"].to(torch.complex128), sto["theta_hat"])
    assert err < 2e-5, err


def test_deterministic_replay(P):
    g = P.make_grid(256, TWO_PI)
    s = P.gSQGSolver(g, 1.0, 0.0, 8, precision="float32", scheme="ifrk4")
    ring = P.RingForcing(20.0, 2.0, 0.1)
    damp = P.CombinedDamping(0.1, 20.0, 1e-12, 8)
    rng = np.random.default_rng(1)
    noise = ring.draw_phases(rng, g, n_steps=5)
    st0 = s.initialize(seed=3)
    a = s.multistep(st0, 5, 1e-3, forcing=ring, damping=damp, noise=noise)
    b = s.multistep(st0, 5, 1e-3, forcing=ring, damping=damp, noise=noise)
    assert torch.equal(a["theta_hat"], b["theta_hat"])


def test_nonfinite_detected(P):
    from pygsquig_b200.exceptions import NumericalError

    g = P.make_grid(32, TWO_PI)
    s = P.gSQGSolver(g, 1.0, 0.0, 8, check_finite=True)
    st = s.initialize(seed=1)
    th = st["theta_hat"].clone()
    th[3, 4] = float("nan")
    with pytest.raises(NumericalError):
        s.step({"theta_hat": th, "time": 0.0, "step": 0}, 1e-3)
    # the solver is still usable afterwards
    s.step(st, 1e-3)


def test_inviscid_energy_conservation(P):
    # test_integration.py:217-246: < 1e-3 over 100 steps, N=64, dt=1e-4
    from pygsquig_b200.utils.diagnostics import compute_total_energy

    g = P.make_grid(64, TWO_PI)
    s = P.gSQGSolver(g, 1.0, 0.0)
    st = s.initialize(seed=333)
    e0 = compute_total_energy(st["theta_hat"], g, 1.0)
    for _ in range(10):
        st = s.multistep(st, 10, 1e-4)
        e = compute_total_energy(st["theta_hat"], g, 1.0)
        assert abs(e - e0) / e0 < 1e-3


@pytest.mark.parametrize("N,prec", [(1024, "float32"), (4096, "float32"), (1024, "float64")])
def test_large_grid_properties(P, N, prec):
    """Full-size cases: finite, multistep == step bit for bit, and the
    inviscid RHS conserves <theta^2> (<theta RHS> = 0, test_solver.py:182-201)."""
    g = P.make_grid(N, TWO_PI)
    s = P.gSQGSolver(g, 0.5, 0.0, 8, precision=prec, scheme="ifrk4")
    k = g.k1d
    x = g.x.cpu().numpy()
    y = g.y.cpu().numpy()
    th0 = np.sin(3 * x) * np.cos(2 * y) + 0.5 * np.cos(5 * x + 1.0) * np.sin(7 * y)
    st = s.initialize(theta0=th0)
    r = s.compute_rhs(st["theta_hat"])
    th = s.plan().to_physical(st["theta_hat"]) if prec == "float64" else None
    tend = s.plan().inner(st["theta_hat"], r)
    assert abs(tend) < (1e-10 if prec == "float64" else 1e-4)
    a = s.multistep(st, 3, 1e-4)
    b = st
    for _ in range(3):
        b = s.step(b, 1e-4)
    assert torch.equal(a["theta_hat"], b["theta_hat"])
    assert torch.isfinite(torch.view_as_real(a["theta_hat"])).all()
