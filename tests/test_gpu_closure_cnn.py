"""Closure CNN on the tensor cores against the float64 oracle: forward
output and every parameter gradient (BF16 activations through five layers:
relative L2 tolerance 3e-2 on the output, 6e-2 on the gradients), and a
short Adam run that must reduce the loss."""

import numpy as np
import pytest
import torch

from oracle import closure_oracle as CO

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_cnn_forward_backward_vs_oracle():
    from pygsquig_b200.build import build

    build()
    from pygsquig_b200.closure.cnn import ClosureCNN

    H, W = 8, 128
    net = ClosureCNN(H=H, W=W, max_batch=2, seed=3)
    rng = np.random.default_rng(4)
    x = rng.standard_normal((2, H, W))
    t = rng.standard_normal((2, H, W)) * 0.1
    xt = torch.as_tensor(x, dtype=torch.float32, device="cuda")
    tt = torch.as_tensor(t, dtype=torch.float32, device="cuda")
    y = net.forward(xt)
    loss = net.mse(y, tt)
    net.backward(xt, net.gy[:2])
    torch.cuda.synchronize()
    assert net.errors() == 0
    p = {k: v.detach().double().cpu().numpy() for k, v in net.p.items()}
    yo, c = CO.forward(p, x)
    go = CO.backward(p, c, 2 * (yo - t) / yo.size)
    assert rel(y.double().cpu().numpy(), yo) < 3e-2
    assert abs(float(loss) - np.mean((yo - t) ** 2)) < 3e-2 * np.mean((yo - t) ** 2)
    for k in p:
        gk = net.g[k].double().cpu().numpy()
        assert rel(gk, go[k]) < 6e-2, (k, rel(gk, go[k]))


def test_cnn_training_reduces_loss():
    from pygsquig_b200.closure.cnn import ClosureCNN

    H, W = 16, 128
    net = ClosureCNN(H=H, W=W, max_batch=2, seed=1)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(2, H, W, device="cuda", generator=g)
    t = torch.roll(x, 1, dims=2) - x  # a learnable local map
    l0 = float(net.train_step(x, t))
    for _ in range(60):
        l1 = float(net.train_step(x, t))
    assert net.errors() == 0
    assert l1 < 0.3 * l0, (l0, l1)
