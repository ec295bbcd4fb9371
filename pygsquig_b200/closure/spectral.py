"""Spectral tools of the closure pipeline: the sharp filter from a DNS grid to
the coarse grid, spectral interpolation to a finer grid, and per-shell
energy spectra / transfer.

Spectra use the solver's convention: the unnormalised (N, N) transform with
axis 0 = kx, on [0, L)^2.  A coefficient divided by N^2 is the physical
Fourier amplitude, so spectra from different grids compare directly.
"""

from __future__ import annotations

import math

import torch


def _fold_index(Nc: int, Nf: int, device) -> torch.Tensor:
    """Index into an Nf-point fft axis of each of the Nc coarse modes."""
    i = torch.arange(Nc, device=device)
    return torch.where(i < Nc // 2, i, i + (Nf - Nc))


def _kmag(N: int, L: float, device) -> torch.Tensor:
    k1 = torch.fft.fftfreq(N, L / N, dtype=torch.float64, device=device) * (2 * math.pi)
    return torch.sqrt(k1[:, None] ** 2 + k1[None, :] ** 2)


class SpectralFilter:
    """Sharp spectral filter of an Nf-grid spectrum onto the Nc grid.

    Keeps the modes with |k| < k_cut (default: the coarse grid's 2/3
    dealiasing radius (2/3) pi Nc / L, so that the filtered field lives where
    the coarse solver's dealiased tendencies live) and rescales by
    (Nc / Nf)^2 to the coarse transform's normalisation.
    """

    def __init__(self, Nf: int, Nc: int, L: float = 2 * math.pi, k_cut: float | None = None, device="cuda"):
        if Nc > Nf or Nf % Nc:
            raise ValueError("the coarse grid must divide the fine grid")
        self.Nf, self.Nc, self.L = Nf, Nc, L
        self.k_cut = (2.0 / 3.0) * math.pi * Nc / L if k_cut is None else k_cut
        self.ix = _fold_index(Nc, Nf, device)
        self.mask = (_kmag(Nc, L, device) < self.k_cut)
        self.scale = (Nc / Nf) ** 2

    def __call__(self, fh: torch.Tensor) -> torch.Tensor:
        sub = fh.index_select(0, self.ix).index_select(1, self.ix)
        return sub * (self.mask * self.scale).to(sub.dtype)


def interpolate_spectrum(ch: torch.Tensor, Nf: int) -> torch.Tensor:
    """Zero-padding interpolation of an Nc-grid spectrum onto the Nf grid (the
    Nyquist row and column of the coarse grid are dropped)."""
    Nc = ch.shape[0]
    ix = _fold_index(Nc, Nf, ch.device)
    keep = torch.ones(Nc, dtype=torch.bool, device=ch.device)
    keep[Nc // 2] = False
    ixk = ix[keep]
    out = torch.zeros((Nf, Nf), dtype=ch.dtype, device=ch.device)
    src = ch[keep][:, keep] * ((Nf / Nc) ** 2)
    out[ixk[:, None], ixk[None, :]] = src
    return out


class ShellSpectrum:
    """Per-integer-shell spectra on an N grid: shell k holds the modes with
    k - 1/2 <= |k| < k + 1/2 (L = 2 pi gives integer wavenumbers).

    energy(th)       E(k) = sum_shell 1/2 |k|^(alpha-2) |th|^2 / N^4
                     (so that sum_k E(k) = 1/2 <psi theta>, psi = |k|^-alpha th);
    transfer(th, n)  T(k) = sum_shell Re(conj(psi) n) / N^4 for a tendency
                     spectrum n; the energy flux through k is -sum_{k' <= k} T.
    All sums run on the device; results are float64 tensors of n_shell.
    """

    def __init__(self, N: int, L: float = 2 * math.pi, alpha: float = 1.0, device="cuda"):
        self.N, self.alpha = N, alpha
        k = _kmag(N, L, device)
        self.shell = torch.floor(k * (L / (2 * math.pi)) + 0.5).long().view(-1)
        self.n_shell = int(self.shell.max().item()) + 1
        ks = torch.where(k > 0, k, torch.ones_like(k))
        self.w_e = (0.5 * ks ** (alpha - 2.0) / float(N) ** 4).view(-1)
        self.w_e[0] = 0.0
        self.w_t = (ks ** (-alpha) / float(N) ** 4).view(-1)
        self.w_t[0] = 0.0

    def _bin(self, vals: torch.Tensor) -> torch.Tensor:
        out = torch.zeros(self.n_shell, dtype=torch.float64, device=vals.device)
        return out.index_add_(0, self.shell, vals)

    def energy(self, th: torch.Tensor) -> torch.Tensor:
        a = th.reshape(-1)
        return self._bin((a.real.double() ** 2 + a.imag.double() ** 2) * self.w_e)

    def transfer(self, th: torch.Tensor, tend: torch.Tensor) -> torch.Tensor:
        a, b = th.reshape(-1), tend.reshape(-1)
        re = a.real.double() * b.real.double() + a.imag.double() * b.imag.double()
        return self._bin(re * self.w_t)
