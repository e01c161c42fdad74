"""The hand-written discrete adjoint of the fused RK4 and reference-RK3 rollouts.

Checked three ways: against torch.fft autograd through the plain torch path
(float64, same arithmetic up to rounding), against central finite differences
of the fused forward (float64), and float32 against float64 at the adjoint
configuration's full size (128^3, 100 steps, checkpoints every 10).  RK3 is
the reference's scheme, SSP3 the corrected SSP-RK3 (parity=False); ETD2 the
corrected ETD2 (its first step RK4), whose reference-weight form has no
adjoint and is refused through the C ABI.
"""
import math

import numpy as np
import pytest
import torch

from sles import _native as nat
from sles.adjoint import ETD2Rollout, RK3Rollout, RK4Rollout, log_spectrum_misfit, shell_spectrum
from sles.plain_torch import PlainSolver
from sles.synthetic import random_spectrum_velocity

pytestmark = pytest.mark.gpu


def _field(n, seed=3, k0=4.0):
    u, v, w = random_spectrum_velocity(n, k0, 1.0, seed=seed)
    return torch.stack([torch.as_tensor(x) for x in (u, v, w)]).to("cuda", torch.float64)


def _rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


_ROLLOUT = {"RK4": RK4Rollout, "RK3": RK3Rollout, "SSP3": RK3Rollout}


def _pair(method, n, nu, dt, les, cs, every):
    """(fused rollout, plain torch solver) of one scheme."""
    parity = method != "SSP3"
    ro = _ROLLOUT[method](n, nu, dt, les=les, Cs=cs, dtype=torch.float64, parity=parity, checkpoint_every=every)
    ps = PlainSolver(n, 3, nu=nu, dt=dt, les=les, Cs=cs, method="RK4" if method == "RK4" else "RK3",
                     parity=parity, device="cuda")
    return ro, ps
_UNSUPPORTED = 2  # SLES_ERR_UNSUPPORTED, include/sles.h


@pytest.mark.parametrize("method", ["RK4", "RK3", "SSP3"])
@pytest.mark.parametrize("les", ["Smagorinsky", "vreman", None])
def test_one_step_vjp_matches_torch_autograd(les, method):
    _one_step_vjp(32, 3e-3, 5e-3, 0.17, les, method)


def test_one_step_vjp_256_matches_torch_autograd():
    """The adjoint z pass on the 256-point grid's z-line plan (128-point
    half-length transforms pairing each bin with its mirror in one thread):
    one RK4 Smagorinsky step, float64."""
    _one_step_vjp(256, 1e-4, 1e-3, 0.17, "Smagorinsky", "RK4")
    torch.cuda.empty_cache()


def _one_step_vjp(n, nu, dt, cs, les, method):
    ro, ps = _pair(method, n, nu, dt, les, cs, 1)
    step = ps.rk4 if method == "RK4" else ps.rk3
    U0 = ps.rfft(_field(n))
    g = torch.Generator(device="cuda").manual_seed(1)
    lam = torch.complex(torch.randn(U0.shape, generator=g, device="cuda", dtype=torch.float64),
                        torch.randn(U0.shape, generator=g, device="cuda", dtype=torch.float64))
    # torch autograd through the plain path
    Ua = U0.clone().requires_grad_(True)
    Ca = torch.tensor(cs, dtype=torch.float64, device="cuda", requires_grad=True)
    La = (torch.conj(lam) * step(Ua, Ca)).real.sum()
    gU_ref, = torch.autograd.grad(La, [Ua], retain_graph=True)
    gC_ref = torch.autograd.grad(La, [Ca])[0] if les else None
    # the fused path and its adjoint
    Ub = U0.clone().requires_grad_(True)
    Cb = torch.tensor(cs, dtype=torch.float64, device="cuda", requires_grad=True)
    UT = ro(Ub, Cb, 1)
    assert _rel(UT.detach(), step(U0).detach()) < 1e-12
    Lb = (torch.conj(lam) * UT).real.sum()
    Lb.backward()
    assert _rel(Ub.grad, gU_ref) < 1e-10
    if les:
        assert abs(float(Cb.grad) - float(gC_ref)) <= 1e-9 * abs(float(gC_ref))


@pytest.mark.parametrize("method", ["RK4", "RK3", "SSP3"])
def test_checkpointed_rollout_matches_torch_autograd(method):
    n, nu, dt, cs, steps = 32, 2e-3, 5e-3, 0.17, 7
    ro, ps = _pair(method, n, nu, dt, "Smagorinsky", cs, 3)
    U0 = ps.rfft(_field(n, seed=4))
    Et = shell_spectrum(U0, n).detach() * 0.9
    Ua = U0.clone().requires_grad_(True)
    Ca = torch.tensor(cs, dtype=torch.float64, device="cuda", requires_grad=True)
    La = log_spectrum_misfit(ps.rollout(Ua, steps, Ca), Et, n)
    La.backward()
    Ub = U0.clone().requires_grad_(True)
    Cb = torch.tensor(cs, dtype=torch.float64, device="cuda", requires_grad=True)
    Lb = log_spectrum_misfit(ro(Ub, Cb, steps), Et, n)
    Lb.backward()
    assert abs(float(La.detach()) - float(Lb.detach())) <= 1e-11 * abs(float(La.detach()))
    assert _rel(Ub.grad, Ua.grad) < 1e-9
    assert abs(float(Cb.grad) - float(Ca.grad)) <= 1e-9 * abs(float(Ca.grad))


def _loss(ro, U0, cs, steps, Et, n):
    with torch.no_grad():
        return float(log_spectrum_misfit(ro(U0, torch.tensor(cs, dtype=torch.float64, device="cuda"), steps),
                                         Et, n))


@pytest.mark.parametrize("les,method", [("Smagorinsky", "RK4"), ("vreman", "RK4"), ("Smagorinsky", "RK3"),
                                        ("vreman", "SSP3")])
def test_gradients_match_central_differences(les, method):
    n, nu, dt, cs, steps = 48, 2e-4, 2e-3, 0.17, 12
    ro = _ROLLOUT[method](n, nu, dt, les=les, Cs=cs, dtype=torch.float64, parity=method != "SSP3",
                          checkpoint_every=5)
    U0 = ro.rfft(_field(n, seed=6))
    Et = shell_spectrum(U0, n).detach() * torch.linspace(0.8, 1.2, shell_spectrum(U0, n).numel(), device="cuda",
                                                         dtype=torch.float64)
    U = U0.clone().requires_grad_(True)
    C = torch.tensor(cs, dtype=torch.float64, device="cuda", requires_grad=True)
    log_spectrum_misfit(ro(U, C, steps), Et, n).backward()
    # C_s: central differences with eps = 1e-3 and 5e-4; their truncation error
    # is O(eps^2) (~1e-4 relative here), the Richardson combination's O(eps^4)
    cd = lambda e: (_loss(ro, U0, cs + e, steps, Et, n) - _loss(ro, U0, cs - e, steps, Et, n)) / (2 * e)
    fd1, fd2 = cd(1e-3), cd(5e-4)
    rich = (4.0 * fd2 - fd1) / 3.0
    assert abs(rich - float(C.grad)) <= 1e-5 * abs(rich)
    assert abs(fd1 - float(C.grad)) <= 1e-3 * abs(fd1)
    # U_hat: random-direction probes (a solenoidal, real-consistent direction)
    g = torch.Generator(device="cuda").manual_seed(7)
    for _ in range(2):
        d = ro.rfft(_field(n, seed=int(torch.randint(100, 1000, (1,), generator=g, device="cuda"))))
        d = d / torch.linalg.vector_norm(d) * torch.linalg.vector_norm(U0)
        h = 1e-5
        fd = (_loss(ro, U0 + h * d, cs, steps, Et, n) - _loss(ro, U0 - h * d, cs, steps, Et, n)) / (2 * h)
        an = float((torch.conj(U.grad) * d).real.sum())
        assert abs(fd - an) <= 1e-5 * abs(fd)


def test_adjoint_configuration_float32_against_float64():
    """128^3 Smagorinsky, RK4, nu=2e-4, dt=2e-3, 100 steps, checkpoints every 10:
    float32 gradients against float64 gradients of the same fused path."""
    n, nu, dt, cs, steps = 128, 2e-4, 2e-3, 0.17, 100
    r64 = RK4Rollout(n, nu, dt, les="Smagorinsky", Cs=cs, dtype=torch.float64, checkpoint_every=10)
    r32 = RK4Rollout(n, nu, dt, les="Smagorinsky", Cs=cs, dtype=torch.float32, checkpoint_every=10)
    U0 = r64.rfft(_field(n, seed=0))
    Et = shell_spectrum(U0, n).detach() * 0.8
    grads = []
    for ro, dtp in ((r64, torch.complex128), (r32, torch.complex64)):
        U = U0.to(dtp).clone().requires_grad_(True)
        C = torch.tensor(cs, dtype=torch.float64, device="cuda", requires_grad=True)
        log_spectrum_misfit(ro(U, C, steps), Et, n, kmax=20).backward()
        grads.append((U.grad.to(torch.complex128), float(C.grad)))
    (g64, c64), (g32, c32) = grads
    assert _rel(g32, g64) < 1e-3
    assert abs(c32 - c64) <= 1e-3 * abs(c64)


@pytest.mark.parametrize("steps,every", [(1, 10), (2, 10), (4, 10), (7, 3)])
@pytest.mark.parametrize("les", ["Smagorinsky", "vreman", None])
def test_etd2_rollout_matches_torch_autograd(les, steps, every):
    n, nu, dt, cs = 32, 3e-3, 5e-3, 0.17
    ro = ETD2Rollout(n, nu, dt, les=les, Cs=cs, dtype=torch.float64, checkpoint_every=every)
    ps = PlainSolver(n, 3, nu=nu, dt=dt, les=les, Cs=cs, method="ETD2", parity=False, device="cuda")
    U0 = ps.rfft(_field(n, seed=8))
    g = torch.Generator(device="cuda").manual_seed(2)
    lam = torch.complex(torch.randn(U0.shape, generator=g, device="cuda", dtype=torch.float64),
                        torch.randn(U0.shape, generator=g, device="cuda", dtype=torch.float64))
    Ua = U0.clone().requires_grad_(True)
    Ca = torch.tensor(cs, dtype=torch.float64, device="cuda", requires_grad=True)
    ps.first = True
    out = Ua
    for _ in range(steps):
        out = ps.step(out, Ca)
    La = (torch.conj(lam) * out).real.sum()
    gU_ref, = torch.autograd.grad(La, [Ua], retain_graph=True)
    gC_ref = torch.autograd.grad(La, [Ca])[0] if les else None
    Ub = U0.clone().requires_grad_(True)
    Cb = torch.tensor(cs, dtype=torch.float64, device="cuda", requires_grad=True)
    UT = ro(Ub, Cb, steps)
    assert _rel(UT.detach(), out.detach()) < 1e-12
    (torch.conj(lam) * UT).real.sum().backward()
    assert _rel(Ub.grad, gU_ref) < 1e-10
    if les:
        assert abs(float(Cb.grad) - float(gC_ref)) <= 1e-9 * abs(float(gC_ref))


def test_etd2_gradients_match_central_differences():
    n, nu, dt, cs, steps = 48, 2e-4, 2e-3, 0.17, 12
    ro = ETD2Rollout(n, nu, dt, les="Smagorinsky", Cs=cs, dtype=torch.float64, checkpoint_every=5)
    U0 = ro.rfft(_field(n, seed=6))
    Et = shell_spectrum(U0, n).detach() * torch.linspace(0.8, 1.2, shell_spectrum(U0, n).numel(), device="cuda",
                                                         dtype=torch.float64)
    U = U0.clone().requires_grad_(True)
    C = torch.tensor(cs, dtype=torch.float64, device="cuda", requires_grad=True)
    log_spectrum_misfit(ro(U, C, steps), Et, n).backward()
    cd = lambda e: (_loss(ro, U0, cs + e, steps, Et, n) - _loss(ro, U0, cs - e, steps, Et, n)) / (2 * e)
    fd1, fd2 = cd(1e-3), cd(5e-4)
    rich = (4.0 * fd2 - fd1) / 3.0
    assert abs(rich - float(C.grad)) <= 1e-5 * abs(rich)
    d = ro.rfft(_field(n, seed=123))
    d = d / torch.linalg.vector_norm(d) * torch.linalg.vector_norm(U0)
    h = 1e-5
    fd = (_loss(ro, U0 + h * d, cs, steps, Et, n) - _loss(ro, U0 - h * d, cs, steps, Et, n)) / (2 * h)
    an = float((torch.conj(U.grad) * d).real.sum())
    assert abs(fd - an) <= 1e-5 * abs(fd)


@pytest.mark.parametrize("scheme,parity", [(nat.SCHEME_ETD2, True)])
def test_schemes_without_an_adjoint_are_refused(scheme, parity):
    """The reference's ETD2 weights (parity arithmetic) have no adjoint; the
    adjoint entry points return SLES_ERR_UNSUPPORTED for its plans."""
    n = 32
    plan = nat.Plan(3, n, torch.float64, nat.LES_SMAGORINSKY, scheme, parity, 1e-3, 0.17, 0.0, torch.device("cuda"))
    _, ws = plan.adjoint_workspace()
    z = torch.zeros((3, n, n, plan.nkp), dtype=torch.complex128, device="cuda")
    with pytest.raises(nat.SlesError) as e:
        plan.adjoint_seed(ws, 1e-3, z, z.clone(), z.clone())
    assert e.value.status == _UNSUPPORTED
    csg = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(nat.SlesError) as e:
        plan.adjoint_stage(ws, 0, 1e-3, None, z, z.clone(), z.clone(), csg)
    assert e.value.status == _UNSUPPORTED
    torch.cuda.synchronize()


@pytest.mark.parametrize("method", ["RK4", "RK3", "SSP3", "ETD2"])
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-11), (torch.float32, 1e-4)])
def test_adjoint_x_pass_forms_agree(method, dtype, tol):
    # ETD2: the reverse ETD2 steps load directly under both settings; its first
    # (RK4) step's reverse runs on the companion RK4 plan, which does switch
    """The adjoint x pass through the TMA tile ring (SLES_PASS_AX variant 1, the
    default) against the direct-load form (variant 0): same reverse sweep,
    128^3, 3 steps with checkpoints every 2 (prime, interior and last stages)."""
    n, nu, dt, cs, steps = 128, 1e-3, 2e-3, 0.17, 3
    if method == "ETD2":
        ro = ETD2Rollout(n, nu, dt, les="Smagorinsky", Cs=cs, dtype=dtype, checkpoint_every=2)
        plans = (ro.plan, ro.rk.plan)
    else:
        ro = _ROLLOUT[method](n, nu, dt, les="Smagorinsky", Cs=cs, dtype=dtype, parity=method != "SSP3",
                              checkpoint_every=2)
        plans = (ro.plan,)
    for p in plans:
        assert p.variant_count(nat.PASS_AX) == 2 and p.get_variant(nat.PASS_AX) == 1
    U0 = ro.rfft(_field(n, seed=5))
    UT, ck = ro.forward_states(U0, cs, steps)
    g0 = torch.randn(UT[..., : ro.nk].shape, dtype=ro.rdtype, device="cuda",
                     generator=torch.Generator(device="cuda").manual_seed(1)).to(ro.cdtype)
    out = []
    for v in (0, 1):
        for p in plans:
            p.set_variant(v, nat.PASS_AX)
        g, c = ro.backward_states(ck, g0, cs, steps)
        out.append((g[..., : ro.nk].to(torch.complex128).clone(), float(c)))
    (ga, ca), (gb, cb) = out
    assert _rel(gb, ga) < tol
    assert abs(cb - ca) <= tol * abs(ca)
