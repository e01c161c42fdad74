"""Smagorinsky closure with the reference's entry points (src/smagorinsky.py:8-47)."""
from __future__ import annotations

import torch

from .math_formula import residue_stress, velocity_gradient

__all__ = ["Smagorinsky_model", "calculate_nuR"]


def Smagorinsky_model(domain, dU=None):
    velocity_gradient(domain)
    calculate_nuR(domain)
    domain.temp_I = residue_stress(domain)
    return domain.temp_I


def calculate_nuR(domain):
    """nu_t = (Cs dx)^2 sqrt(2 S:S) (src/smagorinsky.py:24-47)."""
    d = domain
    if d.dim == 3:
        s = (d.a11 * d.a11 + 0.5 * (d.a12 + d.a21) ** 2 + d.a22 * d.a22 + 0.5 * (d.a13 + d.a31) ** 2
             + 0.5 * (d.a23 + d.a32) ** 2 + d.a33 * d.a33)
    else:
        s = d.a11 * d.a11 + 0.5 * (d.a12 + d.a21) ** 2 + d.a22 * d.a22
    d.nuR = torch.sqrt(2.0 * s) * (d.Cs * d.dx) ** 2
