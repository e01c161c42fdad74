"""Full-size checks on the benchmark grids (256^3 and 512^3), through
size-independent properties: the FP32 fused path against the FP64 fused path
(the FP64 kernels are parity-tested against the oracle on small grids) a few
steps in, and a divergence-free state (k . U_hat = 0 to round-off).  Inputs:
the seeded random-phase spectrum (k0 = 4 or 6, u0 = 1).

Tolerances: relative L2 of FP32 against FP64 below 1e-5 after 5 steps (the
stated bound is 1e-4 after 100 steps); |k . U_hat| below 1e-5 of |k| |U_hat|
in L2 for FP32 (1e-12 for FP64).
"""
import math

import pytest
import torch

from sles import ETD2_method, RK3_method
from sles.initial import initial_velocity
from sles.initialize_domain import InitializeDomain
from sles.synthetic import random_spectrum_velocity

pytestmark = pytest.mark.gpu


def _domain(n, dtype, method="RK3", les="Smagorinsky", nu=1e-4, cs=0.17, dt=1e-3, k0=4.0, parity=True, seed=0):
    # the reference's LES grid is No_of_gridpoint / 4 (src/initialize_domain.py:39-40)
    d = InitializeDomain(nu=nu, dimension=3, time_stepSize=dt, No_of_gridpoint=4 * n, method=method, LES_ON=1,
                         LES_model=les, Cs=cs, dtype=dtype, parity_mode=parity)
    u, v, w = random_spectrum_velocity(n, k0, 1.0, seed=seed)
    initial_velocity(d, u, v, w)
    return d


def _rel(a, b):
    return float(torch.linalg.vector_norm(a.to(b.dtype) - b) / torch.linalg.vector_norm(b))


def _divergence(U, n):
    """||k . U|| / || |k| |U| || over the stored half-complex modes."""
    dev = U.device
    rd = torch.float64
    kc = (torch.fft.fftfreq(n, device=dev, dtype=rd) * n).round()
    kz = torch.arange(n // 2 + 1, device=dev, dtype=rd)
    K = [kc.view(n, 1, 1), kc.view(1, n, 1), kz.view(1, 1, -1)]
    num = den = 0.0
    for x in range(0, n, 64):  # slabs of x, to bound the temporaries
        s = slice(x, x + 64)
        Us = [U[c, s].to(torch.complex128) for c in range(3)]
        div = K[0][s] * Us[0] + K[1] * Us[1] + K[2] * Us[2]
        kk = torch.sqrt(K[0][s] ** 2 + K[1] ** 2 + K[2] ** 2)
        mag = kk * torch.sqrt(sum(u.real ** 2 + u.imag ** 2 for u in Us))
        num += float((div.real ** 2 + div.imag ** 2).sum())
        den += float((mag ** 2).sum())
    return math.sqrt(num / den)


def _release():
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("n", [256, 512])
def test_smagorinsky_rk3_float32_against_float64(n):
    """The Smagorinsky recipe on the benchmark grids (reference RK3, Cs = 0.17,
    nu = 1e-4, dt = 1e-3)."""
    d32, d64 = _domain(n, "float32"), _domain(n, "float64")
    for _ in range(5):
        RK3_method.solveForNextTimestep(d32)
        RK3_method.solveForNextTimestep(d64)
    d32._plan.check()
    d64._plan.check()
    assert torch.isfinite(d32.U_hat).all()
    assert _rel(d32.U_hat, d64.U_hat) < 1e-5
    assert _divergence(d32.U_hat, n) < 1e-5
    assert _divergence(d64.U_hat, n) < 1e-12
    del d32, d64
    _release()


def test_vreman_etd2_512_float32_against_float64():
    """The Vreman ETD2 case at 512^3 (k0 = 6, nu = 5e-5, c = 0.07 i.e.
    Cs = sqrt(0.028), dt = 5e-4, corrected ETD2)."""
    n, cs = 512, math.sqrt(0.07 / 2.5)
    mk = lambda dt_: _domain(n, dt_, method="ETD2", les="vreman", nu=5e-5, cs=cs, dt=5e-4, k0=6.0, parity=False)
    d32, d64 = mk("float32"), mk("float64")
    for _ in range(5):
        ETD2_method.solveForNextTimestep(d32)
        ETD2_method.solveForNextTimestep(d64)
    d32._plan.check()
    d64._plan.check()
    assert _rel(d32.U_hat, d64.U_hat) < 1e-5
    assert _divergence(d32.U_hat, n) < 1e-5
    del d32, d64
    _release()
