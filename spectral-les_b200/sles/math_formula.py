"""Spectral operators with the reference's signatures (src/math_formula.py),
computed on the GPU through the domain's transforms.  The steppers do not use
these: they run the fused kernels.  Provided so code written against the
reference's helpers keeps working."""
from __future__ import annotations

import torch

__all__ = ["U_cross_omega", "del_cross_U", "velocity_gradient", "residue_stress"]


def _kt(K, like):
    return torch.as_tensor(K, device=like.device)


def U_cross_omega(fft, dim, a, b, c):
    """c = rfftn(a x b) (src/math_formula.py:5-13)."""
    if dim == 2:
        c[0] = fft.forward(a[1] * b)
        c[1] = fft.forward(-a[0] * b)
    else:
        c[0] = fft.forward(a[1] * b[2] - a[2] * b[1])
        c[1] = fft.forward(a[2] * b[0] - a[0] * b[2])
        c[2] = fft.forward(a[0] * b[1] - a[1] * b[0])
    return c


def del_cross_U(fft, dim, a, c, K):
    """c = irfftn(i K x a) (src/math_formula.py:16-25)."""
    K = _kt(K, a)
    if dim == 2:
        c[...] = fft.backward(1j * (K[0] * a[1] - K[1] * a[0]))
    else:
        c[2] = fft.backward(1j * (K[0] * a[1] - K[1] * a[0]))
        c[1] = fft.backward(1j * (K[2] * a[0] - K[0] * a[2]))
        c[0] = fft.backward(1j * (K[1] * a[2] - K[2] * a[1]))
    return c


_NAMES3 = [["a11", "a12", "a13"], ["a21", "a22", "a23"], ["a31", "a32", "a33"]]


def velocity_gradient(domain):
    """a_ij = irfftn(i K_i U_hat_j) stored as domain.a11 ... (src/math_formula.py:27-62)."""
    d = domain
    g = torch.empty((d.dim * d.dim,) + d.shape, dtype=d._rdtype, device=d.device)
    d._plan.velocity_gradient(d._s_uhat, g)
    d._primed = None
    for i in range(d.dim):
        for j in range(d.dim):
            setattr(d, _NAMES3[i][j], g[i * d.dim + j])
    return


def residue_stress(domain):
    """temp_I = 2i * dealias * sum_j K_j rfftn(nuR S_ij) (src/math_formula.py:64-146,
    including the reference's 2D component-0 overwrite)."""
    d = domain
    K = _kt(d.K, d._U)
    mask = torch.as_tensor(d.dealias, device=d.device)
    A = [[getattr(d, _NAMES3[i][j]) for j in range(d.dim)] for i in range(d.dim)]
    S = lambda i, j: A[i][i] if i == j else 0.5 * (A[i][j] + A[j][i])
    nuR = d.nuR
    if not hasattr(d, "temp_I") or d.temp_I is None:
        d.temp_I = torch.zeros_like(d.U_hat)
    if d.dim == 3:
        for i in range(3):
            acc = 0
            for j in range(3):
                acc = acc + K[j] * d.fft.forward(S(i, j) * nuR)
            d.temp_I[i] = acc * (2.0 * 1j * mask)
    else:
        d.temp_I[0] = (K[0] * d.fft.forward(S(0, 1) * nuR) + K[1] * d.fft.forward(S(1, 1) * nuR)) * (2.0 * 1j * mask)
    return d.temp_I
