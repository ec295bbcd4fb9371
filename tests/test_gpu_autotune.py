"""Launch-shape autotuning of the transform passes: every shape gives
bit-identical results (forced, damped IF-RK4 steps, ring forcing included),
and the tuner picks a valid shape."""

import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,prec", [(64, "float64"), (256, "float32"), (256, "float64"), (512, "float32")])
def test_every_shape_gives_identical_steps(N, prec):
    from pygsquig_b200 import CombinedDamping, RingForcing, gSQGSolver, make_grid
    from pygsquig_b200.build import build

    build()
    g = make_grid(N, 2 * math.pi)
    s = gSQGSolver(g, 1.0, 0.0, 8, precision=prec, scheme="ifrk4")
    ring = RingForcing(N / 8, 2.0, 0.1)
    damp = CombinedDamping(0.1, N / 8, 1e-12, 8)
    rng = np.random.default_rng(1)
    st0 = s.initialize(theta0=rng.standard_normal((N, N)))
    noise = torch.as_tensor(rng.uniform(0, 2 * math.pi, (3, ring.n_modes(g))), device="cuda")
    pl = s.plan(damp, ring)
    sh = pl.shape()
    assert sh["rpc"] <= sh["max_rpc"] and sh["np"] <= sh["max_np"]
    ref = None
    r = sh["max_rpc"]
    while r >= 1:
        n = sh["max_np"]
        while n >= 1:
            pl.set_shape(r, n)
            out = s.multistep(st0, 3, 1e-3, forcing=ring, damping=damp, noise=noise)["theta_hat"]
            if ref is None:
                ref = out
            else:
                assert torch.equal(out, ref), (r, n)
            n //= 2
        r //= 2
    pl.autotune()
    with pytest.raises(ValueError):
        pl.set_shape(3, 0)
