"""Forcing plug-ins on the host (no GPU): constructor validation of the
deterministic and stochastic forcings (the reference's ForcingError cases),
and the stochastic generators against a NumPy restatement drawn from the
same numpy Generator (they build their noise wherever theta_hat lives)."""

import math

import numpy as np
import pytest
import torch

from pygsquig_b200 import make_grid
from pygsquig_b200.exceptions import ForcingError
from pygsquig_b200.forcing import (
    CheckerboardForcing,
    ColoredNoiseForcing,
    CombinedDeterministicForcing,
    KolmogorovForcing,
    OrnsteinUhlenbeckForcing,
    ShearLayerForcing,
    StochasticVortexForcing,
    TaylorGreenForcing,
    TimeModulatedForcing,
    VortexPairForcing,
    WhiteNoiseForcing,
    create_combined_stochastic_forcing,
    make_oscillating_forcing,
)

G = make_grid(32, 2 * math.pi)


@pytest.mark.parametrize("make", [
    lambda: TaylorGreenForcing(amplitude=0), lambda: TaylorGreenForcing(k=0), lambda: TaylorGreenForcing(k=1.5),
    lambda: KolmogorovForcing(direction="z"), lambda: CheckerboardForcing(ky=0),
    lambda: ShearLayerForcing(profile="cubic"), lambda: ShearLayerForcing(width=0),
    lambda: VortexPairForcing([(0, 0, 1)]), lambda: VortexPairForcing([(0, 0, 1, -1)]),
    lambda: VortexPairForcing([], amplitude_scale=0), lambda: TimeModulatedForcing(object()),
    lambda: TimeModulatedForcing(KolmogorovForcing(), modulation="square"),
    lambda: TimeModulatedForcing(KolmogorovForcing(), frequency=0), lambda: CombinedDeterministicForcing([(1, 2)]),
    lambda: make_oscillating_forcing("spiral"), lambda: WhiteNoiseForcing(amplitude=-1),
    lambda: ColoredNoiseForcing(amplitude=-1), lambda: StochasticVortexForcing(vortex_size=2),
    lambda: StochasticVortexForcing(injection_rate=-1), lambda: OrnsteinUhlenbeckForcing(correlation_time=0),
    lambda: create_combined_stochastic_forcing([]),
    lambda: create_combined_stochastic_forcing([WhiteNoiseForcing()], weights=[1, 2]),
    lambda: create_combined_stochastic_forcing([WhiteNoiseForcing()], weights=[0]),
])
def test_validation(make):
    with pytest.raises(ForcingError):
        make()


def _kmag():
    return np.sqrt(G.kx.cpu().numpy() ** 2 + G.ky.cpu().numpy() ** 2)


def _corners(z):
    z = z.copy()
    for i, j in ((0, 0), (16, 0), (0, 16), (16, 16)):
        z[i, j] = z[i, j].real
    return z


def test_white_noise_matches_numpy():
    th = torch.zeros(32, 32, dtype=torch.complex128)
    f = WhiteNoiseForcing(amplitude=0.3, k_min=2.0, k_max=9.0)
    got = f(th, np.random.default_rng(4), 0.01, G).numpy()
    rng = np.random.default_rng(4)
    z = (rng.standard_normal((32, 32)) + 1j * rng.standard_normal((32, 32))) * 0.3 * math.sqrt(0.01)
    k = _kmag()
    m = (k >= 2.0) * (k <= 9.0) * 1.0
    m[0, 0] = 0
    z = _corners(z * m)
    z *= math.sqrt(0.3**2 * 0.01 / (np.sum(np.abs(z) ** 2) / 32**4))
    z[0, 0] = 0
    np.testing.assert_allclose(got, z, rtol=1e-13, atol=0)
    assert math.isclose(np.sum(np.abs(got) ** 2) / 32**4, 0.3**2 * 0.01, rel_tol=1e-12)
    assert all(got[i, j].imag == 0 for i, j in ((16, 0), (0, 16), (16, 16)))


def test_colored_noise_matches_numpy():
    th = torch.zeros(32, 32, dtype=torch.complex64)
    f = ColoredNoiseForcing(amplitude=0.2, spectral_slope=-2.0, k_peak=6.0, k_width=3.0)
    got = f(th, np.random.default_rng(9), 0.04, G)
    assert got.dtype == torch.complex64
    rng = np.random.default_rng(9)
    z = rng.standard_normal((32, 32)) + 1j * rng.standard_normal((32, 32))
    k = _kmag()
    ks = np.where(k > 0, k, 1.0)
    s = np.where(k > 0, (ks / 6.0) ** -2.0 * np.exp(-(((ks - 6.0) / 3.0) ** 2)), 0.0)
    z = _corners(z * np.sqrt(s) * 0.2 * math.sqrt(0.04))
    z[0, 0] = 0
    np.testing.assert_allclose(got.numpy(), z.astype(np.complex64), rtol=1e-5, atol=1e-7)


def test_ou_recursion():
    th = torch.zeros(32, 32, dtype=torch.complex128)
    f = OrnsteinUhlenbeckForcing(amplitude=0.5, correlation_time=0.2, k_max=8.0)
    rng_a, rng_b = np.random.default_rng(1), np.random.default_rng(1)
    n0 = rng_b.standard_normal((32, 32))
    state = n0 + 1j * n0
    k = _kmag()
    m = (k <= 8.0) * 1.0
    m[0, 0] = 0
    for _ in range(3):
        got = f(th, rng_a, 0.05, G).numpy()
        e = math.exp(-0.05 / 0.2)
        n = rng_b.standard_normal((32, 32))
        state = e * state + 0.5 * math.sqrt(2 * 0.05 / 0.2 * (1 - e**2)) * (n + 1j * n)
        ref = _corners(state * m)
        ref[0, 0] = 0
        np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-15)


def test_combined_stochastic_weights():
    th = torch.zeros(32, 32, dtype=torch.complex128)
    a, b = WhiteNoiseForcing(amplitude=0.1), WhiteNoiseForcing(amplitude=0.2)
    c = create_combined_stochastic_forcing([a, b], weights=[1, 3])
    got = c(th, np.random.default_rng(2), 0.01, G)
    rng = np.random.default_rng(2)
    fa = a(th, rng, 0.01, G)
    fb = b(th, rng, 0.01, G)
    assert torch.allclose(got, 0.25 * fa + 0.75 * fb, rtol=1e-14, atol=0)
    assert c.weights == [0.25, 0.75]


def test_time_modulation_advances_per_call():
    class Unit(TaylorGreenForcing):
        def __call__(self, theta_hat, key, dt, grid):
            return torch.ones(2, dtype=torch.complex128)

    for mod, fn in (("sine", lambda t: math.sin(2 * math.pi * 2.0 * t + 0.3)),
                    ("cosine", lambda t: math.cos(2 * math.pi * 2.0 * t + 0.3)),
                    ("exponential", lambda t: math.exp(-0.7 * t)), ("ramp", lambda t: min(0.7 * t, 1.0))):
        f = TimeModulatedForcing(Unit(), modulation=mod, frequency=2.0, decay_rate=0.7, phase=0.3)
        for i in range(4):
            out = f(None, None, 0.5, G)
            assert math.isclose(out[0].real, fn(0.5 * i), rel_tol=1e-15, abs_tol=1e-15)
        assert f._time == 2.0
