"""RK3 (src/RK3_method.py).  parity_mode=True reproduces the reference's
scheme, which with its single dU buffer reduces to U0 + dt*k3
(src/RK3_method.py:26-33); parity_mode=False runs SSP-RK3."""
from __future__ import annotations

from . import _stepper
from .diagnostics import U_square, dissipation_rate  # noqa: F401  (src/RK3_method.py:83-107)

__all__ = ["solveForNextTimestep", "computeRHS", "U_square", "dissipation_rate"]


def solveForNextTimestep(domain):
    _stepper.rk3_step(domain)


def computeRHS(domain, dU, rk):
    """src/RK3_method.py:44-77 (identical to RK4's)."""
    return _stepper.compute_rhs(domain, dU, rk)
