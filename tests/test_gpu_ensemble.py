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


def _mixed_members(rng, sizes_counts, n_scal_max=3):
    from pygsquig_b200.ensemble import Member

    out = []
    for N, count in sizes_counts:
        g = O.make_grid(N, TWO_PI)
        for _ in range(count):
            alpha = float(rng.choice([0.0, 0.5, 1.0, 1.5]))
            th0 = O.random_phase_field(g, lambda k: (k / 8.0) ** 4 * np.exp(-2 * (k / 8.0) ** 2),
                                       int(rng.integers(1 << 30)))
            ns = int(rng.integers(0, n_scal_max + 1))
            sc = [blob(N, *rng.uniform(0, TWO_PI, 2)) for _ in range(ns)]
            out.append(Member(N, alpha, th0, sc, [float(rng.choice([1e-4, 1e-3]))] * ns))
    return out


@pytest.mark.parametrize("prec,use_graph", [("float64", True), ("float32", True), ("float64", False)])
def test_unified_launches_match_class_by_class(prec, use_graph):
    """Sizes 128, 256 and 512 in one launch per pass (scalars pipelined one
    step behind theta) against the same members stepped class by class."""
    from pygsquig_b200.build import build

    build()
    from pygsquig_b200.ensemble import EnsembleSolver

    rng = np.random.default_rng(11)
    members = _mixed_members(rng, [(128, 3), (256, 2), (512, 2)])
    members[0].scalars0, members[0].kappa = [blob(128, 1.0, 2.0)], [1e-3]  # at least one scalar
    nu, dt, n = 1e-6, 5e-4, 5
    uni = EnsembleSolver(members, nu_p=nu, p=8, precision=prec, scheme="ifrk4")
    ref = EnsembleSolver(members, nu_p=nu, p=8, precision=prec, scheme="ifrk4", unified=False)
    assert uni.unified is not None and ref.unified is None
    uni.multistep(n, dt, use_graph=use_graph)
    ref.multistep(n, dt, use_graph=True)
    torch.cuda.synchronize()
    tol = 1e-12 if prec == "float64" else 2e-6
    for i in range(len(members)):
        a, b = uni.state(i), ref.state(i)
        e = (torch.linalg.norm(a["theta_hat"] - b["theta_hat"]) / torch.linalg.norm(b["theta_hat"])).item()
        assert e < tol, (i, e)
        for q in range(len(members[i].scalars0)):
            e = (torch.linalg.norm(a["scalars"][q] - b["scalars"][q]) / torch.linalg.norm(b["scalars"][q])).item()
            assert e < tol, (i, q, e)
    # one launch per pass: 8 per fused step, plus the input pass, theta's
    # first step and the scalars' last step
    assert uni.launches_per_step() == pytest.approx((1 + 8 + 8 * (n - 1) + 8) / n)
    assert ref.launches_per_step() > 3 * uni.launches_per_step()


def test_unified_members_vs_oracle():
    """One member of each size (128, 256, 512), with scalars, through the
    unified launches against the float64 oracle's gSQGSolverWithScalars
    (IF-RK4; the scalars use theta's new velocity): <= 1e-11 after 4 steps."""
    from pygsquig_b200.build import build

    build()
    from pygsquig_b200.ensemble import EnsembleSolver, Member

    rng = np.random.default_rng(3)
    members = []
    for N, alpha in ((128, 0.5), (256, 1.0), (512, 1.5)):
        g = O.make_grid(N, TWO_PI)
        th0 = O.random_phase_field(g, lambda k: (k / 8.0) ** 4 * np.exp(-2 * (k / 8.0) ** 2), N)
        members.append(Member(N, alpha, th0, [blob(N, *rng.uniform(0, TWO_PI, 2)) for _ in range(2)], [1e-3, 1e-4]))
    nu, dt, n = 1e-6, 5e-4, 4
    ens = EnsembleSolver(members, nu_p=nu, p=8, precision="float64", scheme="ifrk4")
    assert ens.unified is not None
    ens.multistep(n, dt)
    torch.cuda.synchronize()
    for i, m in enumerate(members):
        g = O.make_grid(m.N, TWO_PI)
        so = O.gSQGSolverWithScalars(g, m.alpha, nu, 8, passive_scalars={f"s{q}": {"kappa": k} for q, k in
                                                                         enumerate(m.kappa)}, scheme="ifrk4")
        st = so.initialize(theta0=m.theta0, scalar_init={f"s{q}": f for q, f in enumerate(m.scalars0)})
        for _ in range(n):
            st = so.step(st, dt)
        got = ens.state(i)
        th = got["theta_hat"].cpu().numpy()
        e = np.linalg.norm(th - st["theta_hat"]) / np.linalg.norm(st["theta_hat"])
        assert e < 1e-11, (m.N, e)
        for q in range(2):
            sq = got["scalars"][q].cpu().numpy()
            ref = st["scalars"][f"s{q}"]
            e = np.linalg.norm(sq - ref) / np.linalg.norm(ref)
            assert e < 1e-11, (m.N, q, e)
