"""Deterministic and stochastic forcing on the GPU: each pattern's spectrum
against NumPy's FFT of the same physical pattern, and an RK4 step of the
solver with the forcing in its spectral-term slot against the float64
oracle's RK4 with the same term added at every stage."""

import math

import numpy as np
import pytest
import torch

from oracle import sqg_oracle as O
from pygsquig_b200 import gSQGSolver, make_grid
from pygsquig_b200.forcing import (
    CheckerboardForcing,
    ColoredNoiseForcing,
    CombinedDeterministicForcing,
    KolmogorovForcing,
    OrnsteinUhlenbeckForcing,
    ShearLayerForcing,
    StochasticVortexForcing,
    TaylorGreenForcing,
    VortexPairForcing,
    WhiteNoiseForcing,
)

pytestmark = pytest.mark.gpu
N, L = 64, 2 * math.pi


@pytest.fixture(scope="module", autouse=True)
def _built():
    from pygsquig_b200.build import build

    build()


def _xy():
    x1 = np.arange(N) * (L / N)
    return np.meshgrid(x1, x1, indexing="ij")


def _periodic(d):
    d = np.where(d > L / 2, d - L, d)
    return np.where(d < -L / 2, d + L, d)


CASES = [
    (lambda: TaylorGreenForcing(amplitude=0.7, k=3),
     lambda x, y: 0.7 * np.sin(3 * x) * np.cos(3 * y)),
    (lambda: KolmogorovForcing(amplitude=2.0, k=4, direction="x"), lambda x, y: 2.0 * np.sin(4 * x)),
    (lambda: CheckerboardForcing(amplitude=0.5, kx=2, ky=3),
     lambda x, y: 0.5 * np.sign(np.sin(2 * x) * np.sin(3 * y))),
    (lambda: ShearLayerForcing(amplitude=1.5, profile="tanh", direction="y", width=0.4),
     lambda x, y: 1.5 * np.tanh((y - L / 2) / 0.4)),
    (lambda: ShearLayerForcing(amplitude=1.0), lambda x, y: y / L - 0.5),
    (lambda: VortexPairForcing([(1.0, 2.0, 1.0, 0.3), (5.5, 0.2, -0.5, 0.5)], amplitude_scale=2.0),
     lambda x, y: 2.0 * (1.0 / (math.pi * 0.09) * np.exp(-(_periodic(x - 1.0) ** 2 + _periodic(y - 2.0) ** 2) / 0.09)
                         - 0.5 / (math.pi * 0.25) * np.exp(-(_periodic(x - 5.5) ** 2 + _periodic(y - 0.2) ** 2) / 0.25))),
]


@pytest.mark.parametrize("i", range(len(CASES)))
def test_pattern_spectra(i):
    make, pattern = CASES[i]
    g = make_grid(N, L)
    x, y = _xy()
    ref = np.fft.fft2(pattern(x, y))
    th = torch.zeros(N, N, dtype=torch.complex128, device="cuda")
    got = make()(th, None, 0.01, g).cpu().numpy()
    assert np.linalg.norm(got - ref) <= 1e-12 * max(np.linalg.norm(ref), 1.0)
    got32 = make()(th.to(torch.complex64), None, 0.01, g)
    assert got32.dtype == torch.complex64


def test_combined_and_diagnostics():
    g = make_grid(N, L)
    a, b = TaylorGreenForcing(amplitude=1.0, k=2), KolmogorovForcing(amplitude=1.0, k=3)
    c = CombinedDeterministicForcing([(0.5, a), (2.0, b)])
    th = torch.zeros(N, N, dtype=torch.complex128, device="cuda")
    f = c(th, None, 0.1, g)
    assert torch.allclose(f, 0.5 * a(th, None, 0.1, g) + 2.0 * b(th, None, 0.1, g))
    s = gSQGSolver(g, 1.0, 0.0, 8)
    st = s.initialize(seed=4)
    d = c.get_diagnostics(st["theta_hat"], f, g)
    theta = np.real(np.fft.ifft2(st["theta_hat"].cpu().numpy()))
    force = np.real(np.fft.ifft2(f.cpu().numpy()))
    assert math.isclose(d["injection_rate"], float(np.mean(theta * force)), rel_tol=1e-10, abs_tol=1e-14)
    assert d["n_components"] == 2 and d["forcing_type"] == "CombinedDeterministicForcing"


@pytest.mark.parametrize("precision,tol", [("float64", 1e-12), ("float32", 2e-5)])
def test_forced_step_matches_oracle(precision, tol):
    g = make_grid(N, L)
    kol = KolmogorovForcing(amplitude=0.8, k=3)
    s = gSQGSolver(g, 1.0, 1e-12, 8, precision=precision)
    st = s.initialize(seed=2)
    dt = 2e-3
    th0 = st["theta_hat"].to(torch.complex128).cpu().numpy()
    og = O.make_grid(N, L)
    x, y = _xy()
    F = np.fft.fft2(0.8 * np.sin(3 * y))
    ref = th0
    for _ in range(3):
        st = s.step(st, dt, forcing=lambda th, **kw: kol(th, None, dt, g))
        ref = O.rk4_step(ref, lambda t: O.core_rhs(t, og, 1.0, 1e-12, 8) + F, dt)
    got = st["theta_hat"].to(torch.complex128).cpu().numpy()
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < tol, err


def test_stochastic_on_device_generator():
    g = make_grid(N, L)
    th = torch.zeros(N, N, dtype=torch.complex64, device="cuda")
    gen = torch.Generator(device="cuda").manual_seed(5)
    for f in (WhiteNoiseForcing(amplitude=0.2, k_max=10.0), ColoredNoiseForcing(),
              OrnsteinUhlenbeckForcing(k_min=2.0)):
        out = f(th, gen, 0.01, g)
        assert out.device.type == "cuda" and out.dtype == torch.complex64 and out[0, 0] == 0
        assert all(out[i, j].imag == 0 for i, j in ((N // 2, 0), (0, N // 2), (N // 2, N // 2)))
    # the same seed gives the same noise
    a = WhiteNoiseForcing()(th, torch.Generator(device="cuda").manual_seed(9), 0.01, g)
    b = WhiteNoiseForcing()(th, torch.Generator(device="cuda").manual_seed(9), 0.01, g)
    assert torch.equal(a, b)


def test_stochastic_vortex_matches_numpy():
    g = make_grid(N, L)
    f = StochasticVortexForcing(amplitude=0.3, vortex_size=0.05, injection_rate=400.0)
    th = torch.zeros(N, N, dtype=torch.complex128, device="cuda")
    got = f(th, np.random.default_rng(8), 0.01, g).cpu().numpy()
    rng = np.random.default_rng(8)
    n = rng.poisson(4.0)
    assert n > 0
    xs, ys = rng.random(n) * L, rng.random(n) * L
    st = 0.3 * (1 + 0.2 * rng.standard_normal(n))
    sg = 2.0 * (rng.random(n) < 0.5) - 1.0
    x, y = _xy()
    R2 = (0.05 * L) ** 2
    phys = sum(st[i] * sg[i] * np.exp(-((x - xs[i]) ** 2 + (y - ys[i]) ** 2) / (2 * R2)) for i in range(n))
    ref = np.fft.fft2(phys)
    assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)
