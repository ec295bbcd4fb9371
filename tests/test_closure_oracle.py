"""The float64 closure-CNN oracle: analytic gradients against central finite
differences (no GPU)."""

import numpy as np

from oracle import closure_oracle as CO


def params(rng, scale=0.2):
    p = {"w1": rng.standard_normal((9, 64)) * scale, "b1": rng.standard_normal(64) * 0.1,
         "w6": rng.standard_normal((9, 64)) * scale * 0.2, "b6": rng.standard_normal(1) * 0.1}
    for l in range(2, 6):
        p[f"w{l}"] = rng.standard_normal((9, 64, 64)) * scale * 0.15
        p[f"b{l}"] = rng.standard_normal(64) * 0.1
    return p


def test_oracle_gradients_finite_differences():
    rng = np.random.default_rng(0)
    p = params(rng)
    x = rng.standard_normal((1, 4, 5))
    t = rng.standard_normal((1, 4, 5))
    loss = lambda pp: np.mean((CO.forward(pp, x)[0] - t) ** 2)  # noqa: E731
    y, c = CO.forward(p, x)
    g = CO.backward(p, c, 2 * (y - t) / y.size)
    for name, idx in [("w1", (4, 7)), ("b1", (3,)), ("w3", (2, 5, 9)), ("b4", (10,)), ("w5", (8, 1, 63)),
                      ("w6", (0, 12)), ("b6", (0,)), ("w2", (4, 33, 2))]:
        h = 1e-6
        pp = {k: v.copy() for k, v in p.items()}
        pp[name][idx] += h
        lp = loss(pp)
        pp[name][idx] -= 2 * h
        lm = loss(pp)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[name][idx]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (name, fd, g[name][idx])
