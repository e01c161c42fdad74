"""Float64 diagnostics on the GPU.

``energy``/``dissipation``/``spectrum`` use Parseval on U_hat with
compensated float64 sums; ``U_square`` and ``dissipation_rate`` keep the
reference's definitions (src/RK4_method.py:77-101: sum of mean(u_i^2) without
the 1/2, and nu * sum (not mean) of u . irfftn(K^2 U_hat));
``reference_binned_spectrum`` is the reference's width-5 mean binning
(src/SM_solver.py:94-192).
"""
from __future__ import annotations

import math

import numpy as np
import torch

__all__ = ["diag", "energy", "dissipation", "spectrum", "max_velocity", "U_square", "dissipation_rate",
           "reference_binned_spectrum"]


def diag(domain, with_max=False, nshell=0):
    """Device-side reduction: returns (E, eps, umax, nonfinite, spectrum or None)."""
    d = domain
    out = torch.zeros(4, dtype=torch.float64, device=d.device)
    spec = torch.zeros(nshell, dtype=torch.float64, device=d.device) if nshell else None
    up = d.U if with_max else None
    d._plan.diag(d._s_uhat, out, up, spec)
    o = out.cpu().numpy()
    return float(o[0]), float(o[1]), float(o[2]), bool(o[3]), (spec.cpu().numpy() if spec is not None else None)


def energy(domain):
    """E = 1/2 <u . u>."""
    return diag(domain)[0]


def dissipation(domain):
    """eps = nu <|grad u|^2> (= 2 nu <S:S> for solenoidal periodic fields)."""
    return diag(domain)[1]


def spectrum(domain, nshell=None):
    """E(k) on integer shells round(|k|), k = 0 .. nshell-1."""
    d = domain
    if nshell is None:
        nshell = int(0.5 * d.N * math.sqrt(d.dim)) + 2
    return diag(domain, nshell=nshell)[4]


def max_velocity(domain):
    """max over components and points of U (signed, as find_max_velocity)."""
    return diag(domain, with_max=True)[2]


def U_square(domain):
    """sum_i mean(U_i^2) (src/RK4_method.py:77-84)."""
    d = domain
    U = d.U.to(torch.float64)
    return float(torch.sum(U * U).item() / d.N ** d.dim)


def dissipation_rate(domain):
    """nu * sum_i sum_x U_i irfftn(K2 U_hat_i) (src/RK4_method.py:87-101), via
    Parseval: = N^d * nu <|grad u|^2>."""
    d = domain
    return dissipation(d) * float(d.N ** d.dim)


def reference_binned_spectrum(domain):
    """(temp_k, temp_Ek) of the reference's calculate_Ek on one rank."""
    d = domain
    avg = 5
    K2 = d.K2
    k2u = np.unique(K2)
    ns = int(round(math.sqrt(np.max(k2u)))) // avg
    Uh = d.U_hat.to(torch.complex128)
    Ek = torch.sum(Uh.real ** 2 + Uh.imag ** 2, 0).cpu().numpy()
    if d.dim == 2:
        Ek[:, 1:] *= 2
    else:
        Ek[:, :, 1:] *= 2
    tk = np.zeros(ns + 1)
    tE = np.zeros(ns + 1)
    for i in range(ns + 1):
        lo, hi = (i * avg) ** 2, ((i + 1) * avg) ** 2
        if np.any(k2u[(k2u >= lo) & (k2u < hi)]):
            sel = (K2 >= lo) & (K2 < hi)
            tk[i] = np.mean(np.sqrt(K2[sel]))
            tE[i] = np.mean(Ek[sel])
    return tk, tE
