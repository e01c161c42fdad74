"""Vreman closure with the reference's entry points (src/vreman.py:8-147)."""
from __future__ import annotations

import torch

from .math_formula import residue_stress, velocity_gradient

__all__ = ["Vreman_model", "calculate_nuR"]


def Vreman_model(domain, dU=None):
    velocity_gradient(domain)
    calculate_nuR(domain)
    domain.temp_I = residue_stress(domain)
    return domain.temp_I


def calculate_nuR(domain):
    """nu_t = sqrt(B_beta) [aa > 1e-4 and sqrt(B_beta) > aa/1e7] sqrt(1/aa)
    * 2.5 Cs^2 dx^2 (src/vreman.py:30-147)."""
    d = domain
    if d.dim == 3:
        a = [[d.a11, d.a12, d.a13], [d.a21, d.a22, d.a23], [d.a31, d.a32, d.a33]]
    else:
        if d.parity_mode:
            raise AttributeError("'InitializeDomain' object has no attribute 'aTemp' "
                                 "(the reference allocates aTemp only in 3D)")
        a = [[d.a11, d.a12], [d.a21, d.a22]]
    n = d.dim
    b = [[sum(a[m][p] * a[m][q] for m in range(n)) for q in range(n)] for p in range(n)]
    if n == 3:
        B = (b[0][0] * b[1][1] - b[0][1] * b[0][1] + b[0][0] * b[2][2] - b[0][2] * b[0][2]
             + b[1][1] * b[2][2] - b[1][2] * b[1][2])
    else:
        B = b[0][0] * b[1][1] - b[0][1] * b[0][1]
    nu = torch.sqrt(B)
    aa = sum(a[i][j] * a[i][j] for i in range(n) for j in range(n))
    d.aTemp = aa
    gate = torch.where((aa > 10e-5) & (nu > aa / 10e6), torch.sqrt(1 / aa), torch.zeros_like(aa))
    d.nuR = nu * gate * (2.5 * d.Cs * d.Cs * d.dx * d.dx)
