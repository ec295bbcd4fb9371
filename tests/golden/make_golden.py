"""Generate golden fixtures by running the reference package itself.

Run in the build container, where the reference source tree is mounted:

    python tests/golden/make_golden.py /root/reference

JAX is not installed there, so ``jax_stand_in`` registers a NumPy-backed
stand-in for the JAX API subset the hot-path modules use; the reference's own
Python code (grid.py, operators.py, solver.py, time_integrator.py,
solver_optimized.py, ring_forcing.py, damping.py, passive_scalar.py,
solver_with_scalars.py, utils/diagnostics.py, scalars/diagnostics.py) is then
imported unmodified and executed on seeded inputs drawn with
``numpy.random.default_rng``.  Ring-forcing noise is injected by replacing
``RingForcing._generate_random_phases`` with a function that returns the
host-drawn phase array, which is the injection point the reference exposes.

Outputs go to ``tests/golden/*.npz`` (small: N <= 32).  The fixtures are what
the oracle and the CUDA path are pinned against; the reference itself is not
needed afterwards.
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import jax_stand_in  # noqa: E402


def smooth_field(grid_x, grid_y, rng, n_modes=6, kmax=5):
    th = np.zeros_like(grid_x)
    for _ in range(n_modes):
        kx, ky = rng.integers(-kmax, kmax + 1, size=2)
        a, ph = rng.standard_normal(), rng.uniform(0, 2 * np.pi)
        th = th + a * np.cos(kx * grid_x + ky * grid_y + ph)
    return th


def main(ref_root: str) -> None:
    jax_stand_in.install()
    sys.path.insert(0, ref_root)

    from pygsquig.core import grid as rgrid
    from pygsquig.core.solver import gSQGSolver
    from pygsquig.core.solver_optimized import gSQGSolverOptimized
    from pygsquig.core.solver_with_scalars import gSQGSolverWithScalars
    from pygsquig.forcing.damping import CombinedDamping
    from pygsquig.forcing.ring_forcing import RingForcing
    from pygsquig.scalars.diagnostics import compute_scalar_variance
    from pygsquig.utils import diagnostics as rdiag

    out = {}
    A = np.asarray

    # 1. grids -------------------------------------------------------------
    for N, L in [(16, 2 * np.pi), (32, 2 * np.pi), (32, 1.0)]:
        g = rgrid.make_grid(N, L)
        tag = f"grid_N{N}_L{'2pi' if L != 1.0 else '1'}"
        out[tag] = dict(
            N=N, L=L, kx=A(g.kx), ky=A(g.ky), k2=A(g.k2), dealias_mask=A(g.dealias_mask)
        )

    N = 32
    L = 2 * np.pi
    g = rgrid.make_grid(N, L)
    x, y = A(g.x), A(g.y)

    # 2. RHS for several alpha, with an anti-Hermitian part incl. Nyquist ----
    rng = np.random.default_rng(101)
    th0 = smooth_field(x, y, rng, n_modes=8, kmax=8) + 0.05 * rng.standard_normal((N, N))
    th_hat = np.fft.fft2(th0)
    anti = 1e-3 * (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N)))
    anti = anti - np.conj(np.roll(np.flip(anti, (0, 1)), 1, (0, 1)))  # anti-Hermitian
    th_hat_nh = th_hat + anti
    rhs_cases = {}
    for i, (alpha, nu, p) in enumerate(
        [(1.0, 1e-6, 8), (0.5, 1e-4, 4), (0.0, 0.0, 8), (1.5, 1e-3, 2), (-1.0, 1e-6, 8)]
    ):
        s = gSQGSolver(g, alpha, nu, p)
        rhs = A(s.compute_rhs(th_hat_nh.view(jax_stand_in.ShimArray)))
        u, v = s.compute_velocity(th_hat_nh.view(jax_stand_in.ShimArray))
        rhs_cases[f"case{i}"] = dict(
            alpha=alpha, nu_p=nu, p=p, rhs=rhs, u=A(u), v=A(v)
        )
    out["rhs"] = dict(theta_hat=th_hat_nh, cases=rhs_cases)

    # 3. unforced RK4 steps via gSQGSolver.step ---------------------------
    rng = np.random.default_rng(202)
    th0 = smooth_field(x, y, rng, n_modes=10, kmax=6)
    s = gSQGSolver(g, 1.0, 1e-12, 8)
    st = s.initialize(theta0=th0.view(jax_stand_in.ShimArray))
    traj = [A(st["theta_hat"])]
    diags = [s.get_diagnostics(st)]
    for _ in range(10):
        st = s.step(st, 1e-2)
        traj.append(A(st["theta_hat"]))
        diags.append(s.get_diagnostics(st))
    out["steps_unforced"] = dict(
        theta0=th0, alpha=1.0, nu_p=1e-12, p=8, dt=1e-2, traj=np.stack(traj),
        diag_ke=np.array([d["kinetic_energy"] for d in diags]),
        diag_ens=np.array([d["enstrophy"] for d in diags]),
        diag_max=np.array([d["max_theta"] for d in diags]),
    )

    # 3b. gSQG alpha=0.5 with p=4 viscosity
    s = gSQGSolver(g, 0.5, 1e-5, 4)
    st = s.initialize(theta0=th0.view(jax_stand_in.ShimArray))
    traj = [A(st["theta_hat"])]
    for _ in range(5):
        st = s.step(st, 5e-3)
        traj.append(A(st["theta_hat"]))
    out["steps_alpha05"] = dict(theta0=th0, alpha=0.5, nu_p=1e-5, p=4, dt=5e-3, traj=np.stack(traj))

    # 4. multistep of the optimised solver (unforced) -----------------------
    so = gSQGSolverOptimized(g, 1.0, 1e-12, 8)
    st = so.initialize(theta0=th0.view(jax_stand_in.ShimArray))
    st = so.multistep(st, 6, 1e-2)
    out["multistep"] = dict(theta0=th0, alpha=1.0, nu_p=1e-12, p=8, dt=1e-2, n=6,
                            theta_hat=A(st["theta_hat"]), time=float(A(st["time"])))

    # 5. forced-dissipative steps: RingForcing + CombinedDamping ------------
    def forced_run(tau_f, n_steps, seed, solver_nu):
        rng = np.random.default_rng(seed)
        th0 = smooth_field(x, y, rng, n_modes=10, kmax=8)
        ring = RingForcing(kf=6.0, dk=2.0, epsilon=0.1, tau_f=tau_f)
        damp = CombinedDamping(mu=0.1, kf=6.0, nu_p=1e-10, p=8)
        s = gSQGSolver(g, 1.0, solver_nu, 8)
        st = s.initialize(theta0=th0.view(jax_stand_in.ShimArray))
        mask = np.abs(np.sqrt(A(g.k2)) - 6.0) <= 1.0
        n_ring = int(mask.sum())
        phases = rng.uniform(0, 2 * np.pi, size=(n_steps, n_ring))
        traj = [A(st["theta_hat"])]
        forcings = []
        dt = 5e-3
        for i in range(n_steps):
            full = np.zeros((N, N))
            full[mask] = phases[i]
            ring._generate_random_phases = (
                lambda key, shape, _f=full: np.exp(1j * _f).view(jax_stand_in.ShimArray)
            )
            forcing = lambda th, _r=ring, **kw: _r(th, None, dt, g)  # noqa: E731
            st = s.step(st, dt, forcing=forcing, damping=damp, grid=g)
            traj.append(A(st["theta_hat"]))
            forcings.append(A(ring(st["theta_hat"], None, dt, g)) if tau_f == 0 else np.zeros((N, N)))
        return dict(theta0=th0, phases=phases, traj=np.stack(traj), kf=6.0, dk=2.0, eps=0.1,
                    tau_f=tau_f, mu=0.1, kf_damp=6.0, nu_damp=1e-10, p=8, nu_solver=solver_nu,
                    dt=dt, n_ring=n_ring, forcing_after=np.stack(forcings))

    out["forced"] = forced_run(0.0, 5, 303, 0.0)
    out["forced_dup_nu"] = forced_run(0.0, 3, 304, 1e-10)
    out["forced_ou"] = forced_run(0.05, 3, 305, 0.0)

    # 6. passive scalars ---------------------------------------------------
    rng = np.random.default_rng(404)
    th0 = smooth_field(x, y, rng, n_modes=10, kmax=6)
    blob = lambda cx, cy, w: np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * w**2))  # noqa: E731
    s_init = {"a": blob(2.0, 3.0, 0.6), "b": blob(4.0, 1.5, 0.8)}
    sw = gSQGSolverWithScalars(
        g, 1.0, 1e-12, 8, passive_scalars={"a": {"kappa": 1e-3}, "b": {"kappa": 0.0}}
    )
    st = sw.initialize(theta0=th0.view(jax_stand_in.ShimArray),
                       scalar_init={k: v.view(jax_stand_in.ShimArray) for k, v in s_init.items()})
    ta, tb, tt = [A(st["scalar_state"].scalars["a"])], [A(st["scalar_state"].scalars["b"])], [A(st["theta_hat"])]
    for _ in range(5):
        st = sw.step(st, 1e-2)
        ta.append(A(st["scalar_state"].scalars["a"]))
        tb.append(A(st["scalar_state"].scalars["b"]))
        tt.append(A(st["theta_hat"]))
    var_a = [float(A(compute_scalar_variance(t.view(jax_stand_in.ShimArray)))) for t in ta]
    out["scalars"] = dict(theta0=th0, a0=s_init["a"], b0=s_init["b"], kappa_a=1e-3, kappa_b=0.0,
                          alpha=1.0, nu_p=1e-12, p=8, dt=1e-2, traj_theta=np.stack(tt),
                          traj_a=np.stack(ta), traj_b=np.stack(tb), var_a=np.array(var_a))

    # 7. diagnostics -------------------------------------------------------
    th_hat = np.fft.fft2(th0)
    dd = {}
    for alpha in (1.0, 0.5, 0.0, 1.5):
        kb, Ek = rdiag.compute_energy_spectrum(th_hat.view(jax_stand_in.ShimArray), g, alpha)
        dd[f"a{alpha}"] = dict(
            energy=float(A(rdiag.compute_total_energy(th_hat.view(jax_stand_in.ShimArray), g, alpha))),
            enstrophy=float(A(rdiag.compute_enstrophy(th_hat.view(jax_stand_in.ShimArray), g, alpha))),
            palinstrophy=float(A(rdiag.compute_palinstrophy(th_hat.view(jax_stand_in.ShimArray), g, alpha))),
            k_bins=A(kb), E_k=A(Ek),
        )
    out["diagnostics"] = dict(theta_hat=th_hat, alphas=dd)

    # write ------------------------------------------------------------------
    def flat(prefix, d, acc):
        for k, v in d.items():
            key = f"{prefix}/{k}" if prefix else k
            if isinstance(v, dict):
                flat(key, v, acc)
            else:
                acc[key] = np.asarray(v)
        return acc

    for name, d in out.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **flat("", d, {}))
    with open(os.path.join(HERE, "MANIFEST.json"), "w") as f:
        json.dump(
            {
                "generator": "tests/golden/make_golden.py",
                "reference": "dfielding14/pygSQuiG (imported unmodified; JAX replaced by "
                "tests/golden/jax_stand_in.py, FFT = numpy pocketfft)",
                "files": sorted(f"{n}.npz" for n in out),
            },
            f,
            indent=1,
        )
    print("wrote", len(out), "fixture files")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
