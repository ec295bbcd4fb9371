"""Float64 NumPy oracle of the closure CNN (TEST INFRASTRUCTURE ONLY).

No reference counterpart: the reference has no learned closure.  Six 3x3
convolutions with circular padding (1 -> 64 -> 64 -> 64 -> 64 -> 64 -> 1),
GELU (tanh form) between them; forward and analytic backward.  Parameter layout
matches pygsquig_b200.closure.cnn: w1 [9, 64], wl [9, 64 out, 64 in],
w6 [9, 64], tap t = 3 (dy + 1) + (dx + 1), out[p] = sum_t in[p + off_t].
The analytic gradients are checked against finite differences in the tests.
"""

import numpy as np


GELU_A = np.sqrt(2.0 / np.pi)
GELU_B = 0.044715


def gelu(z):
    """GELU in its tanh form (Hendrycks & Gimpel 2016), the network's activation."""
    return 0.5 * z * (1 + np.tanh(GELU_A * (z + GELU_B * z**3)))


def gelu_grad(z):
    t = np.tanh(GELU_A * (z + GELU_B * z**3))
    return 0.5 * (1 + t) + 0.5 * z * (1 - t * t) * GELU_A * (1 + 3 * GELU_B * z * z)


def shift(x, t):
    """x[b, y + dy, x + dx, ...] with circular wrap (axes 1, 2)."""
    dy, dx = t // 3 - 1, t % 3 - 1
    return np.roll(np.roll(x, -dy, axis=1), -dx, axis=2)


def unshift(x, t):
    dy, dx = t // 3 - 1, t % 3 - 1
    return np.roll(np.roll(x, dy, axis=1), dx, axis=2)


def forward(p, x):
    """x: [B, H, W] -> (y [B, H, W], cache)."""
    c = {"x": x}
    z = sum(shift(x, t)[..., None] * p["w1"][t] for t in range(9)) + p["b1"]
    c["z1"], a = z, gelu(z)
    c["a1"] = a
    for l in range(2, 6):
        z = sum(np.einsum("bhwi,oi->bhwo", shift(a, t), p[f"w{l}"][t]) for t in range(9)) + p[f"b{l}"]
        c[f"z{l}"], a = z, gelu(z)
        c[f"a{l}"] = a
    y = sum(np.einsum("bhwi,i->bhw", shift(a, t), p["w6"][t]) for t in range(9)) + p["b6"][0]
    return y, c


def backward(p, c, gy):
    g = {}
    a5 = c["a5"]
    g["w6"] = np.stack([np.einsum("bhw,bhwi->i", gy, shift(a5, t)) for t in range(9)])
    g["b6"] = np.array([gy.sum()])
    ga = sum(unshift(gy, t)[..., None] * p["w6"][t] for t in range(9))
    for l in range(5, 1, -1):
        gz = ga * gelu_grad(c[f"z{l}"])
        a_prev = c[f"a{l - 1}"]
        g[f"w{l}"] = np.stack([np.einsum("bhwo,bhwi->oi", gz, shift(a_prev, t)) for t in range(9)])
        g[f"b{l}"] = gz.sum(axis=(0, 1, 2))
        ga = sum(np.einsum("bhwo,oi->bhwi", unshift(gz, t), p[f"w{l}"][t]) for t in range(9))
    gz = ga * gelu_grad(c["z1"])
    g["w1"] = np.stack([np.einsum("bhwo,bhw->o", gz, shift(c["x"], t)) for t in range(9)])
    g["b1"] = gz.sum(axis=(0, 1, 2))
    return g
