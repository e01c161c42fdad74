"""Seeded synthetic initial fields (the reference ships none).

``random_spectrum_velocity``: solenoidal random-phase velocity with
E(k) = 16 sqrt(2/pi) u0^2 k^4/k0^5 exp(-2 k^2/k0^2).  Phases come from
``numpy.random.default_rng(seed)`` on the host (so any implementation that
draws them the same way sees the same field); amplitudes, the projection
u - k (k.u)/k^2, the shell rescale and the inverse transform run on the GPU in
float64.  ``gaussian_vorticity_2d``: Gaussian random vorticity with spectrum
(k/kp)^2 exp(-(k/kp)^2), zero mean, unit rms.
"""
from __future__ import annotations

import math

import numpy as np
import torch

__all__ = ["random_spectrum_velocity", "gaussian_vorticity_2d", "taylor_green"]


def _model_spectrum(k, k0, u0):
    return 16.0 * math.sqrt(2.0 / math.pi) * u0 * u0 * k ** 4 / k0 ** 5 * torch.exp(-2.0 * k * k / (k0 * k0))


def _kgrid(n, device):
    kc = torch.fft.fftfreq(n, 1.0 / n, device=device, dtype=torch.float64).round()
    kr = kc[: n // 2 + 1].clone()
    kr[-1] = -kr[-1]
    return kc.view(n, 1, 1), kc.view(1, n, 1), kr.view(1, 1, -1)


def random_spectrum_velocity(n, k0=4.0, u0=1.0, seed=0, device="cuda"):
    """(u, v, w) float64 device tensors of shape (n, n, n)."""
    kx, ky, kz = _kgrid(n, device)
    K2 = kx * kx + ky * ky + kz * kz
    kmag = torch.sqrt(K2)
    kmax = 2.0 / 3.0 * (n // 2 + 1)
    inside = (kx.abs() < kmax) & (ky.abs() < kmax) & (kz.abs() < kmax)
    nyq = (kx.abs() == n // 2) | (ky.abs() == n // 2) | (kz.abs() == n // 2)
    live = inside & (K2 > 0) & ~nyq
    safe = torch.where(live, kmag, torch.ones_like(kmag))
    amp = torch.where(live, torch.sqrt(_model_spectrum(safe, k0, u0) / (2 * math.pi * safe ** 2)),
                      torch.zeros_like(kmag))
    rng = np.random.default_rng(seed)
    phase = torch.as_tensor(rng.uniform(0.0, 2 * np.pi, size=(3,) + tuple(amp.shape)), device=device)
    uh = amp[None] * torch.exp(1j * phase)
    uh = torch.fft.rfftn(torch.fft.irfftn(uh, s=(n, n, n), dim=(1, 2, 3)), dim=(1, 2, 3))
    kk = torch.where(K2 == 0, torch.ones_like(K2), K2)
    kdotu = kx * uh[0] + ky * uh[1] + kz * uh[2]
    uh = torch.stack([uh[0] - kx * kdotu / kk, uh[1] - ky * kdotu / kk, uh[2] - kz * kdotu / kk])
    uh = uh * live[None]
    w = torch.where((kz > 0) & (kz < n // 2), 2.0, 1.0)
    shell = torch.round(kmag).to(torch.int64).expand(uh.shape[1:])
    e_mode = (0.5 * torch.sum(uh.real ** 2 + uh.imag ** 2, 0) * w).reshape(-1)
    # shell sums on the host: bincount with weights is sequential there (on the
    # GPU it accumulates with atomics, whose order, and so the last bits of
    # every field made from it, changes from call to call)
    e_shell = torch.bincount(shell.reshape(-1).cpu(), weights=e_mode.cpu()).to(device)
    target = _model_spectrum(torch.arange(e_shell.numel(), device=device, dtype=torch.float64), k0, u0)
    scale = torch.where(e_shell > 0, torch.sqrt(target / torch.where(e_shell > 0, e_shell, torch.ones_like(e_shell))),
                        torch.zeros_like(e_shell))
    uh = uh * scale[shell][None]
    u = torch.fft.irfftn(uh, s=(n, n, n), dim=(1, 2, 3)) * float(n) ** 3
    return u[0], u[1], u[2]


def taylor_green(n, device="cuda"):
    x = torch.arange(n, device=device, dtype=torch.float64) * (2 * math.pi / n)
    X, Y, Z = torch.meshgrid(x, x, x, indexing="ij")
    u = torch.sin(X) * torch.cos(Y) * torch.cos(Z)
    v = -torch.cos(X) * torch.sin(Y) * torch.cos(Z)
    return u, v, torch.zeros_like(u)


def gaussian_vorticity_2d(n, seed=0, kp=10.0, device="cuda"):
    kc = torch.fft.fftfreq(n, 1.0 / n, device=device, dtype=torch.float64).round()
    kr = kc[: n // 2 + 1].clone()
    kr[-1] = -kr[-1]
    kx, ky = kc.view(n, 1), kr.view(1, -1)
    k = torch.sqrt(kx * kx + ky * ky)
    rng = np.random.default_rng(seed)
    shape = (n, n // 2 + 1)
    g = torch.as_tensor(rng.standard_normal(shape) + 1j * rng.standard_normal(shape), device=device)
    wh = g * (k / kp) ** 2 * torch.exp(-(k / kp) ** 2)
    nyq = (kx.abs() == n // 2) | (ky.abs() == n // 2)
    wh = torch.where(nyq, torch.zeros_like(wh), wh)
    wh[0, 0] = 0
    w = torch.fft.irfftn(wh, s=(n, n))
    w = w - w.mean()
    return w / torch.sqrt(torch.mean(w * w))
