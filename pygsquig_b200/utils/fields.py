"""Seeded initial fields, drawn on the host (the solver takes them as
``initialize(theta0=...)``)."""

from __future__ import annotations

from typing import Callable

import numpy as np


def random_phase_field(N: int, L: float, spectrum: Callable[[np.ndarray], np.ndarray], seed: int,
                       rms: float = 1.0) -> np.ndarray:
    """Real (N, N) field with uniform random phases (numpy default_rng(seed))
    and shell spectrum |theta(k)|^2 ~ spectrum(|k|): the amplitude of each
    mode is sqrt(spectrum(k) / (2 pi k)) (isotropic shell density), the real
    part of the inverse transform is taken and rescaled to the target rms."""
    k1 = np.fft.fftfreq(N, L / N) * 2 * np.pi
    k = np.sqrt(k1[:, None] ** 2 + k1[None, :] ** 2)
    ks = np.where(k > 0, k, 1.0)
    amp = np.sqrt(np.maximum(spectrum(ks), 0.0) / (2 * np.pi * ks))
    amp[0, 0] = 0.0
    ph = np.random.default_rng(seed).uniform(0.0, 2 * np.pi, size=(N, N))
    th = np.fft.ifft2(amp * np.exp(1j * ph)).real
    s = np.sqrt(np.mean(th**2))
    return th * (rms / s) if s > 0 else th
