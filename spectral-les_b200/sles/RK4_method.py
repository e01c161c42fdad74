"""Classical RK4 (src/RK4_method.py).  Same entry points as the reference."""
from __future__ import annotations

from . import _stepper
from .diagnostics import U_square, dissipation_rate  # noqa: F401  (src/RK4_method.py:77-101)

__all__ = ["solveForNextTimestep", "computeRHS", "U_square", "dissipation_rate"]


def solveForNextTimestep(domain):
    """One RK4 step (src/RK4_method.py:20-35), each stage one fused launch
    sequence.  As in the reference, U_hat1 must equal U_hat on entry."""
    _stepper.rk4_step(domain)


def computeRHS(domain, dU, rk):
    """dU = P(mask*N_hat + T_hat) [+ f U_hat] - nu K^2 U_hat at the current
    U_hat (src/RK4_method.py:38-71)."""
    return _stepper.compute_rhs(domain, dU, rk)
