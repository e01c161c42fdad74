"""Initial-condition setters (src/initial.py:7-54), on the GPU."""
from __future__ import annotations

import torch

__all__ = ["initial_velocity", "initial_vorticity"]


def initial_velocity(domain, u=0, v=0, w=0):
    """U = (u, v, w); U_hat = rfftn(U) (unscaled); curl = irfftn(i k x U_hat).
    Neither dealiased nor projected, as in src/initial.py:7-18."""
    d = domain
    d._U[0] = d._as_real(u)
    d._U[1] = d._as_real(v)
    if d.dim == 3:
        d._U[2] = d._as_real(w)
    d._plan.fft_r2c(d._U, d._s_uhat, d.dim)
    d._plan.velocity_curl(d._s_uhat, None, d._curl)
    d._primed = None
    d._phys_fresh = True
    d._phys_user = True
    d._phys_ver = (d._U._version, d._curl._version)


def initial_vorticity(domain, omega):
    """Streamfunction phi_hat = rfftn(omega)/K2 with phi_hat[0, 0] = 0,
    U_hat = (i K1 phi_hat, -i K0 phi_hat); curl keeps the given omega and U is
    irfftn(U_hat) (src/initial.py:39-54)."""
    d = domain
    om = d._as_real(omega)
    w_hat = d.fft.forward(om)                       # (N, N[, N]) half-complex
    kx, ky, kz = _k_axes(d)
    K = (kx, ky) if d.dim == 2 else (kx, ky, kz)
    k2 = sum(k * k for k in K)
    phi = w_hat / torch.where(k2 == 0, torch.ones_like(k2), k2).to(d._rdtype)
    phi[0, 0] = 0
    uh = d.U_hat
    uh[0] = 1j * K[1].to(d._rdtype) * phi
    uh[1] = -1j * K[0].to(d._rdtype) * phi
    if d.dim == 3:
        uh[2] = 0
        d._curl[2] = om
    else:
        d._curl[...] = om
    d._plan.fft_c2r(d._s_uhat, d._U, d.dim)
    d._primed = None
    d._phys_fresh = True
    d._phys_user = True
    d._phys_ver = (d._U._version, d._curl._version)


def _k_axes(d):
    """Integer wavenumbers as broadcastable device tensors (kx, ky, kz); the
    last axis is the r2c axis with its Nyquist entry at +N/2."""
    n = d.N
    kc = torch.fft.fftfreq(n, 1.0 / n, device=d.device).round().to(torch.int64)
    kr = torch.arange(n // 2 + 1, device=d.device, dtype=torch.int64)
    if d.dim == 3:
        return kc.view(n, 1, 1), kc.view(1, n, 1), kr.view(1, 1, -1)
    return kc.view(n, 1), kr.view(1, -1), None
