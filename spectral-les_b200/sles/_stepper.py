"""Stage sequencing shared by the integrator modules.

Each stage is one ``sles_stage`` call: the fused RHS evaluation plus the
integrator's update, ending with the inverse x-transforms of the new state so
the next stage starts primed.  Buffers change roles instead of being copied
(the reference copies U_hat into U_hat0 at the start of a step,
src/RK4_method.py:21).
"""
from __future__ import annotations

from . import _native as nat


# kernels launched by stage() calls since the last reset (counted, not sampled)
LAUNCHES = [0]


def _key(s):
    return (s.data_ptr(), s._version)


def stage(d, k, dt, ucur, u0, u1, uout, aux=None, flags=0, first=False):
    uphys = cphys = None
    if first:
        uphys, cphys = d._phys_override()
    primed = d._primed == _key(ucur)
    f = flags | (nat.STAGE_PRIMED if primed else 0)
    if d._dtctl is not None:  # dt from the device-side controller (SM_solver device mode)
        d._plan.stage_ctl(k, d._dtctl, d._parity, ucur, u0, u1, uout, aux, uphys, cphys, f)
    else:
        d._plan.stage(k, dt, ucur, u0, u1, uout, aux, uphys, cphys, f)
    LAUNCHES[0] += (4 if d.dim == 3 else 2) + (0 if primed else 1)
    d._primed = None if (flags & nat.STAGE_NO_PREPARE) else _key(uout)


def rk4_step(d, record_f1=False):
    """src/RK4_method.py:20-35.  U_hat1 must equal U_hat on entry."""
    A, B, C = d._s_uhat, d._s_u0, d._s_u1
    dt = d.dt
    for rk in range(4):
        ucur = A if rk == 0 else B
        aux = d._s_f1 if (record_f1 and rk == 3) else None
        flags = nat.STAGE_RK4 | (nat.STAGE_RECORD_F1 if aux is not None else 0)
        stage(d, rk, dt, ucur, A, C, B, aux, flags, first=(rk == 0))
    d._s_uhat, d._s_u0 = B, A
    d._mark_stepped()
    d._parity ^= 1


def rk3_step(d):
    """src/RK3_method.py:20-41 (parity) or SSP-RK3 (parity_mode=False)."""
    A, B = d._s_uhat, d._s_u0
    dt = d.dt
    for rk in range(3):
        stage(d, rk, dt, A if rk == 0 else B, A, None, B, first=(rk == 0))
    d._s_uhat, d._s_u0 = B, A
    d._mark_stepped()
    d._parity ^= 1


def etd2_step(d):
    """src/ETD2_method.py:7-37.  First call: RK4 step recording F1 (parity) or
    RK4 after F1 = N(u_0) (corrected).  Later calls: exponential step."""
    if d.firstIteration:
        if d.parity_mode:
            rk4_step(d, record_f1=True)
        else:  # corrected: F1 = the explicit term (projected u x omega [+ stress] [+ forcing])
            uphys, cphys = d._phys_override()
            tmp = d._new_hc(d.dim)
            d._plan.rhs(d._s_uhat, tmp, d._s_f1, uphys, cphys)
            d._primed = None
            rk4_step(d)
        d.firstIteration = False
        return
    if d.forcing > 0 and d.parity_mode:
        # src/ETD2_method.py:47-50 reads domain.epsilon, which the reference never sets;
        # the corrected scheme treats the forcing explicitly (in F1)
        raise AttributeError("'InitializeDomain' object has no attribute 'epsilon'")
    U = d._s_uhat
    stage(d, 0, d.dt, U, None, d._s_f1, U, d._s_f0, 0, first=True)
    d._s_f0, d._s_f1 = d._s_f1, d._s_f0
    d._mark_stepped()
    d._parity ^= 1


def compute_rhs(d, dU, rk):
    """src/RK4_method.py:38-71: dU at the current U_hat.  rk == 0 uses the
    stored U and curl, rk > 0 derives them from U_hat."""
    uphys = cphys = None
    if rk == 0:
        uphys, cphys = d._phys_override()
    f1 = d._s_f1 if d.method == "ETD2" else None
    du = d._hc_view(d._s_du) if d._s_du is not None else d.dU
    d._plan.rhs(d._s_uhat, d._s_du, f1, uphys, cphys)
    d._primed = None
    if rk > 0:
        d._mark_stepped()
    if dU is not None and dU.data_ptr() != du.data_ptr():
        dU[...] = du
        return dU
    return du
