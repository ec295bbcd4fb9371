"""What the trained closure gains over the coarse solve without it.

Uses the committed network (pygsquig_b200/closure/trained/, made by
``python -m pygsquig_b200.closure.experiment``) and fixtures from the same
run (tests/golden/closure_fixture.npz: four held-out (theta, Pi) pairs of the
filtered N = 2048 DNS, one filtered DNS state, the time-mean filtered DNS
spectrum).

* A priori: on held-out pairs the network's subgrid term is closer to the
  true one than no term at all (relative MSE below 1, positive correlation).
* A posteriori: from the filtered DNS state, 500 coarse steps (0.5 time
  units, about 3 eddy times) with the closure keep the resolved small scales
  (40 <= k < 85) near the DNS spectrum, while the coarse solve without it
  piles energy up there (its error is at least twice the closure's).
"""

import math
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
FIX = os.path.join(HERE, "golden", "closure_fixture.npz")
W = os.path.join(ROOT, "pygsquig_b200", "closure", "trained", "closure_weights.npz")


def _closure():
    from pygsquig_b200.build import build

    build()
    from pygsquig_b200.closure.model import SubgridClosure

    return SubgridClosure.load(W)


def test_a_priori_gain_on_held_out_pairs():
    clo = _closure()
    z = np.load(FIX)
    pl = clo.plan
    num = den = dot = npp = 0.0
    for th, pi in zip(z["theta"], z["pi"]):
        th_hat = pl.to_spectral(torch.as_tensor(th, device="cuda"))
        y = clo.physical(th_hat).double().cpu().numpy()
        num += np.sum((y - pi) ** 2)
        den += np.sum(pi.astype(np.float64) ** 2)
        dot += np.sum(y * pi)
        npp += np.sum(y**2)
    assert clo.errors() == 0
    rel_mse, corr = num / den, dot / math.sqrt(den * npp)
    assert rel_mse < 0.95, rel_mse
    assert corr > 0.3, corr


def test_a_posteriori_small_scales_vs_no_closure():
    from pygsquig_b200.closure import experiment as X
    from pygsquig_b200.closure.model import ClosureSolver
    from pygsquig_b200.closure.spectral import ShellSpectrum

    clo = _closure()
    z = np.load(FIX)
    cfg = X.Config()
    n, m = 500, int(round(cfg.dt_c / cfg.dt))
    shell = ShellSpectrum(cfg.N_c, 2 * math.pi, cfg.alpha)
    E_dns = z["E_dns"]
    k = np.arange(40, 85)
    errs = {}
    for name, c in (("closure", clo), ("none", None)):
        g, s, damp, ring = X._solver(cfg, cfg.N_c, cfg.nu)
        runner = ClosureSolver(s, c, damp, ring, forcing_substeps=m)
        noise = torch.as_tensor(np.random.default_rng(3).uniform(0, 2 * math.pi, (n * m, ring.n_modes(g))),
                                device="cuda")
        st = {"theta_hat": torch.as_tensor(z["ic"], device="cuda"), "time": 0.0, "step": 0}
        E = np.zeros_like(E_dns)
        st = runner.multistep(st, n - 50, cfg.dt_c, noise)  # 450 steps
        for i in range(5):  # the last 50 steps, sampled every 10
            st = runner.multistep(st, 10, cfg.dt_c, noise[(n - 50 + 10 * i) * m:])
            E += shell.energy(st["theta_hat"]).cpu().numpy() / 5
        assert bool(torch.isfinite(torch.view_as_real(st["theta_hat"])).all())
        errs[name] = float(np.mean(np.abs(np.log(E[k] / E_dns[k]))))
    assert clo.errors() == 0
    assert errs["closure"] < 0.5 * errs["none"], errs
