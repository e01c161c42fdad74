"""ETD2 (src/ETD2_method.py).  The first step is RK4.  parity_mode=True
reproduces the reference (its F1 weight (1+hL)/(hL^2) and the LES stress left
out after step 1, src/ETD2_method.py:16-29, 39-46); parity_mode=False uses the
Cox & Matthews (2002) weights, evaluated in float64, with the LES stress in
the nonlinear term."""
from __future__ import annotations

from . import _stepper

__all__ = ["solveForNextTimestep", "computeFn_for_ETD2"]


def solveForNextTimestep(domain):
    _stepper.etd2_step(domain)


def computeFn_for_ETD2(domain):
    """F0 <- F1; F1 <- P(mask * rfftn(u x omega)) at the current state
    (src/ETD2_method.py:39-57).  Provided for API parity; the stepper fuses it."""
    d = domain
    if d.forcing > 0:
        raise AttributeError("'InitializeDomain' object has no attribute 'epsilon'")
    d.F0[...] = d.F1
    tmp = d._new_hc(d.dim)
    uphys, cphys = d._phys_override()
    plan = d._plan
    # the reference's F1 is the projected u x omega term without the LES stress
    if d.LES_ON and d.parity_mode:
        from . import _native as nat
        p2 = nat.Plan(d.dim, d.N, d._rdtype, nat.LES_NONE, nat.SCHEME_ETD2, True, d.nu, d.Cs, 0.0, d.device)
        p2.rhs(d._s_uhat, tmp, d._s_f1, uphys, cphys)
    else:
        plan.rhs(d._s_uhat, tmp, d._s_f1, uphys, cphys)
    d._primed = None
