"""Pin the CPU oracle against fixtures produced by the reference package.

The fixtures in tests/golden were produced by ``tests/golden/make_golden.py``,
which imports the unmodified reference modules (JAX replaced by a NumPy
stand-in).  These tests run without a GPU.
"""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from oracle import sqg_oracle as O  # noqa: E402

GOLD = os.path.join(ROOT, "tests", "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("tag,N,L", [("grid_N16_L2pi", 16, 2 * np.pi), ("grid_N32_L2pi", 32, 2 * np.pi),
                                     ("grid_N32_L1", 32, 1.0)])
def test_grid_bitexact(tag, N, L):
    d = load(tag)
    g = O.make_grid(N, L)
    for k in ("kx", "ky", "k2", "dealias_mask"):
        assert np.array_equal(getattr(g, k), d[k]), k


def test_rhs_cases():
    d = load("rhs")
    g = O.make_grid(32, 2 * np.pi)
    th = d["theta_hat"]
    for i in range(5):
        c = f"cases/case{i}/"
        alpha, nu, p = float(d[c + "alpha"]), float(d[c + "nu_p"]), int(d[c + "p"])
        s = O.gSQGSolver(g, alpha, nu, p)
        assert rel(s.compute_rhs(th), d[c + "rhs"]) < 1e-14
        u, v = s.compute_velocity(th)
        assert rel(u, d[c + "u"]) < 1e-14 and rel(v, d[c + "v"]) < 1e-14


def test_unforced_steps():
    d = load("steps_unforced")
    g = O.make_grid(32, 2 * np.pi)
    s = O.gSQGSolver(g, float(d["alpha"]), float(d["nu_p"]), int(d["p"]))
    st = s.initialize(theta0=d["theta0"])
    for i in range(1, d["traj"].shape[0]):
        st = s.step(st, float(d["dt"]))
        assert rel(st["theta_hat"], d["traj"][i]) < 1e-14
        dg = s.get_diagnostics(st)
        assert abs(dg["kinetic_energy"] - d["diag_ke"][i]) <= 1e-14 * abs(d["diag_ke"][i])
        assert abs(dg["enstrophy"] - d["diag_ens"][i]) <= 1e-14 * abs(d["diag_ens"][i])
        assert abs(dg["max_theta"] - d["diag_max"][i]) <= 1e-14 * abs(d["diag_max"][i])


def test_alpha05_steps():
    d = load("steps_alpha05")
    g = O.make_grid(32, 2 * np.pi)
    s = O.gSQGSolver(g, float(d["alpha"]), float(d["nu_p"]), int(d["p"]))
    st = s.initialize(theta0=d["theta0"])
    for i in range(1, d["traj"].shape[0]):
        st = s.step(st, float(d["dt"]))
        assert rel(st["theta_hat"], d["traj"][i]) < 1e-14


def test_multistep():
    d = load("multistep")
    g = O.make_grid(32, 2 * np.pi)
    s = O.gSQGSolver(g, float(d["alpha"]), float(d["nu_p"]), int(d["p"]))
    st = s.multistep(s.initialize(theta0=d["theta0"]), int(d["n"]), float(d["dt"]))
    assert rel(st["theta_hat"], d["theta_hat"]) < 1e-14
    assert abs(st["time"] - float(d["time"])) < 1e-14


@pytest.mark.parametrize("name", ["forced", "forced_dup_nu", "forced_ou"])
def test_forced_steps(name):
    d = load(name)
    g = O.make_grid(32, 2 * np.pi)
    ring = O.RingForcing(float(d["kf"]), float(d["dk"]), float(d["eps"]), float(d["tau_f"]))
    damp = O.CombinedDamping(float(d["mu"]), float(d["kf_damp"]), float(d["nu_damp"]), int(d["p"]))
    s = O.gSQGSolver(g, 1.0, float(d["nu_solver"]), int(d["p"]))
    st = s.initialize(theta0=d["theta0"])
    assert O.ring_mode_count(g, float(d["kf"]), float(d["dk"])) == int(d["n_ring"])
    for i in range(d["phases"].shape[0]):
        st = O.step_forced(s, st, float(d["dt"]), ring, d["phases"][i], damp)
        assert rel(st["theta_hat"], d["traj"][i + 1]) < 1e-14, i


def test_scalars():
    d = load("scalars")
    g = O.make_grid(32, 2 * np.pi)
    s = O.gSQGSolverWithScalars(g, float(d["alpha"]), float(d["nu_p"]), int(d["p"]),
                                passive_scalars={"a": {"kappa": float(d["kappa_a"])},
                                                 "b": {"kappa": float(d["kappa_b"])}})
    st = s.initialize(theta0=d["theta0"], scalar_init={"a": d["a0"], "b": d["b0"]})
    for i in range(1, d["traj_a"].shape[0]):
        st = s.step(st, float(d["dt"]))
        assert rel(st["theta_hat"], d["traj_theta"][i]) < 1e-14
        assert rel(st["scalars"]["a"], d["traj_a"][i]) < 1e-14
        assert rel(st["scalars"]["b"], d["traj_b"][i]) < 1e-14
        assert abs(O.compute_scalar_variance(st["scalars"]["a"]) - d["var_a"][i]) < 1e-14 * d["var_a"][i]


def test_diagnostics():
    d = load("diagnostics")
    g = O.make_grid(32, 2 * np.pi)
    th = d["theta_hat"]
    for alpha in (1.0, 0.5, 0.0, 1.5):
        c = f"alphas/a{alpha}/"
        assert abs(O.compute_total_energy(th, g, alpha) - d[c + "energy"]) <= 1e-13 * abs(d[c + "energy"])
        assert abs(O.compute_enstrophy(th, g, alpha) - d[c + "enstrophy"]) <= 1e-13 * abs(d[c + "enstrophy"])
        assert abs(O.compute_palinstrophy(th, g, alpha) - d[c + "palinstrophy"]) <= 1e-13 * abs(
            d[c + "palinstrophy"])
        kb, E = O.compute_energy_spectrum(th, g, alpha)
        assert np.allclose(kb, d[c + "k_bins"], rtol=1e-15, atol=0)
        assert np.allclose(E, d[c + "E_k"], rtol=1e-13, atol=1e-300)
