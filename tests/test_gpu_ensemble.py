"""Batched ensembles against the single-field solver, member by member."""

import numpy as np
import pytest
import torch

from oracle import sqg_oracle as O

pytestmark = pytest.mark.gpu
TWO_PI = 2 * np.pi


def blob(N, cx, cy, w=0.3):
    x = np.arange(N) * TWO_PI / N
    X, Y = np.meshgrid(x, x, indexing="ij")
    return np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * w**2))


@pytest.mark.parametrize("prec,use_graph", [("float64", True), ("float32", True), ("float64", False)])
def test_ensemble_members_match_single_solver(prec, use_graph):
    from pygsquig_b200.build import build

    build()
    import pygsquig_b200 as P
    from pygsquig_b200.ensemble import EnsembleSolver, Member

    rng = np.random.default_rng(5)
    specs = [(32, 1.0, 0), (32, 0.5, 2), (64, 0.0, 1), (64, 1.5, 3), (32, 1.0, 1)]
    members = []
    for i, (N, a, ns) in enumerate(specs):
        g = O.make_grid(N, TWO_PI)
        th0 = O.random_phase_field(g, lambda k: k**4 * np.exp(-((k / 4.0) ** 2)), 10 + i)
        sc = [blob(N, *rng.uniform(0, TWO_PI, 2)) for _ in range(ns)]
        members.append(Member(N, a, th0, sc, [1e-3] * ns))
    nu, dt, n = 1e-10, 2e-3, 6
    # FP64: same kernels, differences only from FMA contraction (<= 1e-12);
    # FP32: the single-precision tolerance of the other parity tests
    tol = 1e-12 if prec == "float64" else 2e-6
    ens = EnsembleSolver(members, nu_p=nu, p=8, precision=prec, scheme="ifrk4")
    ens.multistep(n, dt, use_graph=use_graph)
    torch.cuda.synchronize()
    for i, m in enumerate(members):
        g = P.make_grid(m.N, TWO_PI)
        species = {f"s{q}": {"kappa": 1e-3} for q in range(len(m.scalars0))}
        s = P.gSQGSolverWithScalars(g, m.alpha, nu, 8, passive_scalars=species or None, precision=prec,
                                    scheme="ifrk4")
        st = s.initialize(theta0=m.theta0, scalar_init={f"s{q}": f for q, f in enumerate(m.scalars0)})
        for _ in range(n):
            st = s.step(st, dt)
        ref = st["theta_hat"]
        got = ens.state(i)["theta_hat"]
        err = (torch.linalg.norm(got - ref) / torch.linalg.norm(ref)).item()
        assert err < tol, (i, err)
        for q in range(len(m.scalars0)):
            rs = st["scalar_state"].scalars[f"s{q}"]
            gs = ens.state(i)["scalars"][q]
            e = (torch.linalg.norm(gs - rs) / torch.linalg.norm(rs)).item()
            assert e < tol, (i, q, e)
    assert ens.launches_per_step() > 0
