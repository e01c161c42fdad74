"""The benchmark configurations on the GPU, against independent references.

* The plain Taylor-Green case (64^3, RK4, dt = 0.01, nu = 1/1600, no LES,
  float64): the fused path against the oracle after every one of the first
  20 steps (relative L2 of U_hat below 1e-11), then all 200 steps with the
  kinetic energy and dissipation of every step: E(t) against the analytic
  early-time decay E = 1/8 exp(-6 nu t) while t <= 0.2 (the O(t^3) departure
  is 1.05e-6 there in the oracle), and the energy budget dE/dt = -eps to
  2e-5 (central differences of the RK4 steps).
* The Smagorinsky recipe at 256^3 and 512^3 (reference RK3, Cs = 0.17,
  nu = 1e-4, dt = 1e-3, seeded spectrum k0 = 4): the fused float64 and
  float32 paths against the plain torch.fft (cuFFT) float64 path, an
  independent implementation, after 3 steps: relative L2 below 1e-11
  (float64) and 1e-5 (float32; at 512^3 this runs the float32-only y-pass
  geometries: 128-byte tile rows and the 32-thread inverse line plan).
"""
import math

import numpy as np
import pytest
import torch

from oracle import spectral_oracle as so
from sles import RK3_method, RK4_method, diagnostics
from sles.initial import initial_velocity
from sles.initialize_domain import InitializeDomain
from sles.plain_torch import PlainSolver
from sles.synthetic import random_spectrum_velocity

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def test_taylor_green_64_rk4_against_oracle_and_decay():
    n, nu, dt = 64, 1.0 / 1600.0, 0.01
    u = so.taylor_green(n)
    d = InitializeDomain(nu=nu, dimension=3, time_stepSize=dt, No_of_gridpoint=n, method="RK4", dtype="float64")
    initial_velocity(d, *u)
    d.U_hat1[...] = d.U_hat
    o = so.OracleDomain(n, 3, nu=nu, dt=dt, method="RK4")
    so.initial_velocity(o, *u)
    o.U_hat1 = o.U_hat.copy()
    E = [diagnostics.energy(d)]
    eps = [diagnostics.dissipation(d)]
    assert E[0] == pytest.approx(0.125, rel=1e-14)
    for s in range(200):
        RK4_method.solveForNextTimestep(d)
        if s < 20:
            so.step(o)
            err = rel(d.U_hat.cpu().numpy(), o.U_hat)
            assert err < 1e-11, (s + 1, err)
        E.append(diagnostics.energy(d))
        eps.append(diagnostics.dissipation(d))
    d._plan.check()
    E, eps = np.array(E), np.array(eps)
    t = np.arange(E.size) * dt
    exact = 0.125 * np.exp(-6.0 * nu * t)
    early = t <= 0.2 + 1e-12
    assert np.max(np.abs(E[early] - exact[early]) / exact[early]) < 1.5e-6
    dEdt = (E[2:] - E[:-2]) / (2 * dt)
    assert np.max(np.abs(dEdt + eps[1:-1]) / eps[1:-1]) < 2e-5
    assert np.all(np.diff(E) < 0)


def _smag(n, dtype, seed=0):
    d = InitializeDomain(nu=1e-4, dimension=3, time_stepSize=1e-3, No_of_gridpoint=4 * n, method="RK3", LES_ON=1,
                         LES_model="Smagorinsky", Cs=0.17, dtype=dtype)
    u = random_spectrum_velocity(n, 4.0, 1.0, seed=seed)
    initial_velocity(d, *u)
    return d, u


def _trel(a, b):
    num = den = 0.0
    for c in range(a.shape[0]):  # per component, to bound the temporaries
        x = a[c].to(torch.complex128)
        num += float(torch.linalg.vector_norm(x - b[c]) ** 2)
        den += float(torch.linalg.vector_norm(b[c]) ** 2)
    return math.sqrt(num / den)


@pytest.mark.parametrize("n", [256, 512])
def test_fused_against_plain_torch_fp64(n):
    steps = 3
    ps = PlainSolver(n, 3, nu=1e-4, dt=1e-3, les="Smagorinsky", Cs=0.17, method="RK3", parity=True,
                     dtype=torch.float64, device="cuda")
    d, u = _smag(n, "float64")
    Uh = ps.rfft(torch.stack(u))
    del u
    for _ in range(steps):
        Uh = ps.step(Uh)
        RK3_method.solveForNextTimestep(d)
    d._plan.check()
    assert _trel(d.U_hat, Uh) < 1e-11
    del d
    torch.cuda.empty_cache()
    d32, _ = _smag(n, "float32")
    for _ in range(steps):
        RK3_method.solveForNextTimestep(d32)
    d32._plan.check()
    assert _trel(d32.U_hat, Uh) < 1e-5
    del d32, Uh, ps
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("dim,les", [(3, None), (2, "Smagorinsky"), (2, None)])
def test_fused_256_other_forms_against_plain_torch_fp64(dim, les):
    """The 256-point grid's z-line plan (128-point half-length transforms whose
    last stage pairs each bin with its mirror in one thread) in the pass forms
    the Smagorinsky recipe above does not run: 3D without LES and 2D with and
    without Smagorinsky, RK4, float64, 3 steps against the plain torch.fft path
    (relative L2 below 1e-11; 2D LES in the corrected stress form, which the
    plain path implements)."""
    from sles.initial import initial_vorticity
    from sles.synthetic import gaussian_vorticity_2d
    n, steps = 256, 3
    nu = 1e-4 if dim == 3 else 1e-3
    d = InitializeDomain(nu=nu, dimension=dim, time_stepSize=1e-3, No_of_gridpoint=(4 if les else 1) * n,
                         method="RK4", LES_ON=1 if les else 0, LES_model=les, Cs=0.17, dtype="float64",
                         parity_mode=not (dim == 2 and les))
    if dim == 3:
        initial_velocity(d, *random_spectrum_velocity(n, 4.0, 1.0, seed=2))
    else:
        initial_vorticity(d, gaussian_vorticity_2d(n, seed=2, kp=10.0))
    d.U_hat1[...] = d.U_hat
    ps = PlainSolver(n, dim, nu=nu, dt=1e-3, les=les, Cs=0.17, method="RK4", parity=not (dim == 2 and les),
                     dtype=torch.float64, device="cuda")
    Uh = d.U_hat.detach().to(torch.complex128).clone()
    for _ in range(steps):
        Uh = ps.step(Uh)
        RK4_method.solveForNextTimestep(d)
    d._plan.check()
    assert _trel(d.U_hat, Uh) < 1e-11
    del d, ps, Uh
    torch.cuda.empty_cache()
