"""CUDA-graph replay and ensembles give the same state as eager stepping."""
import pytest
import torch

from sles.graph import CapturedStepper, Ensemble
from sles.initial import initial_velocity, initial_vorticity
from sles.initialize_domain import InitializeDomain
from sles.synthetic import gaussian_vorticity_2d, random_spectrum_velocity
from sles.graph import _eager_step

pytestmark = pytest.mark.gpu


def _make(kind, seed):
    if kind == "les3d_rk3":
        d = InitializeDomain(nu=1e-3, dimension=3, time_stepSize=2e-3, No_of_gridpoint=4 * 64, method="RK3",
                             LES_ON=1, LES_model="Smagorinsky", Cs=0.17, dtype="float32")
        initial_velocity(d, *random_spectrum_velocity(64, 4.0, 1.0, seed=seed))
    elif kind == "vreman3d_rk4":
        d = InitializeDomain(nu=1e-3, dimension=3, time_stepSize=2e-3, No_of_gridpoint=4 * 32, method="RK4",
                             LES_ON=1, LES_model="vreman", Cs=0.16733, dtype="float32")
        initial_velocity(d, *random_spectrum_velocity(32, 4.0, 1.0, seed=seed))
    elif kind == "plain3d_etd2":
        d = InitializeDomain(nu=1e-2, dimension=3, time_stepSize=2e-3, No_of_gridpoint=48, method="ETD2",
                             dtype="float32", parity_mode=False)
        initial_velocity(d, *random_spectrum_velocity(48, 4.0, 1.0, seed=seed))
    else:  # 2D vorticity RK4
        d = InitializeDomain(nu=1e-3, dimension=2, time_stepSize=1e-3, No_of_gridpoint=128, method="RK4",
                             dtype="float32")
        initial_vorticity(d, gaussian_vorticity_2d(128, seed=seed))
    d.U_hat1[...] = d.U_hat
    return d


def _rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


@pytest.mark.parametrize("kind,steps", [("les3d_rk3", 8), ("plain3d_etd2", 7), ("vort2d_rk4", 9)])
def test_captured_stepper_matches_eager(kind, steps):
    a, b = _make(kind, 3), _make(kind, 3)
    cs = CapturedStepper(a)
    cs.advance(steps)
    for _ in range(steps):
        _eager_step(b)
    torch.cuda.synchronize()
    assert _rel(a.U_hat, b.U_hat) < 1e-6
    # reading U reuses the workspace; the next advance recaptures and still matches
    assert _rel(a.U, b.U) < 1e-6
    cs.advance(4)
    for _ in range(4):
        _eager_step(b)
    torch.cuda.synchronize()
    assert _rel(a.U_hat, b.U_hat) < 1e-6


def test_ensemble_of_uneven_members_matches_members_alone():
    kinds = ["les3d_rk3", "vreman3d_rk4", "plain3d_etd2", "vort2d_rk4"]
    ens = Ensemble([_make(k, 10 + i) for i, k in enumerate(kinds)])
    solo = [_make(k, 10 + i) for i, k in enumerate(kinds)]
    ens.advance(6)
    for d in solo:
        for _ in range(6):
            _eager_step(d)
    torch.cuda.synchronize()
    for e, s in zip(ens.members, solo):
        assert _rel(e.U_hat, s.U_hat) < 1e-6


def _member(dim, n, dtype, les, method, nu, cs, seed):
    if dim == 3:
        d = InitializeDomain(nu=nu, dimension=3, time_stepSize=1e-3, No_of_gridpoint=(4 if les else 1) * n,
                             method=method, LES_ON=1 if les else 0, LES_model=les, Cs=cs, dtype=dtype)
        initial_velocity(d, *random_spectrum_velocity(n, 4.0, 1.0, seed=seed))
    else:
        d = InitializeDomain(nu=nu, dimension=2, time_stepSize=1e-3, No_of_gridpoint=n, method=method, dtype=dtype)
        initial_vorticity(d, gaussian_vorticity_2d(n, seed=seed))
    d.U_hat1[...] = d.U_hat
    return d


@pytest.mark.parametrize("dtype,tol", [("float64", 1e-12), ("float32", 2e-6)])
def test_member_batches_match_members_alone(dtype, tol):
    """Members of one grid and scheme run as one batched plan (one launch per
    pass, each member's own nu and Cs): the same states as stepping each
    member alone, up to the round-off of the first step (a batch derives U
    and curl from U_hat where a lone domain reuses its setter's fields)."""
    spec = [(3, 32, "Smagorinsky", "RK4", 1e-3, 0.12), (3, 32, "Smagorinsky", "RK4", 2e-4, 0.19),
            (3, 32, "Smagorinsky", "RK4", 5e-4, 0.15), (2, 64, None, "RK4", 1e-5, 0.14),
            (2, 64, None, "RK4", 3e-4, 0.14), (3, 32, "vreman", "RK3", 1e-3, 0.16), (3, 32, "vreman", "RK3", 3e-3, 0.11),
            (3, 48, None, "RK4", 1e-3, 0.14)]
    mk = lambda: [_member(dm, n, dtype, les, me, nu, cs, 20 + i) for i, (dm, n, les, me, nu, cs) in enumerate(spec)]
    ens = Ensemble(mk(), batch=True)
    assert len(ens.batches) == 3 and len(ens.units) == 4
    solo = mk()
    ens.advance(7)
    ens.advance(3)
    for d in solo:
        for _ in range(10):
            _eager_step(d)
    torch.cuda.synchronize()
    for e, s in zip(ens.members, solo):
        assert _rel(e.U_hat, s.U_hat) < tol
