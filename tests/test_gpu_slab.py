"""Slab decomposition kernels on one GPU: the P ranks of one decomposed 3D
domain (sles.slab.SlabDomain, ky rows / x planes as the reference's PFFT
slabs, src/initialize_domain.py:59-65) run in one process, their
all-to-all exchanges done by copies between their buffers
(sles.slab.emulated_exchange), against the whole-grid fused path on the same
field: relative L2 below 1e-12 in float64 and 1e-6 in float32 after 3 steps,
and the same u_max (src/SM_solver.py:245-255).  No rank waits on another:
every exchange is a plain copy between kernel launches.
"""
import pytest
import torch

from sles import RK3_method, RK4_method
from sles.initial import initial_velocity
from sles.initialize_domain import InitializeDomain
from sles.slab import SlabDomain, emulated_exchange
from sles.synthetic import random_spectrum_velocity

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


@pytest.mark.parametrize("n,P,dtype,les,method,tol", [
    (64, 1, "float64", "Smagorinsky", "RK3", 1e-12),
    (64, 2, "float64", "Smagorinsky", "RK3", 1e-12),
    (64, 4, "float64", "vreman", "RK4", 1e-12),
    (32, 2, "float64", None, "RK4", 1e-12),
    (128, 4, "float32", "Smagorinsky", "RK3", 1e-6),
    (256, 2, "float32", "Smagorinsky", "RK3", 1e-6),
    (512, 2, "float32", "Smagorinsky", "RK3", 1e-6),
])
def test_emulated_slab_ranks_match_whole_grid(n, P, dtype, les, method, tol):
    d = InitializeDomain(nu=1e-3, dimension=3, time_stepSize=1e-3, No_of_gridpoint=(4 if les else 1) * n,
                         method=method, LES_ON=1 if les else 0, LES_model=les, Cs=0.17, dtype=dtype)
    initial_velocity(d, *random_spectrum_velocity(n, 4.0, 1.0, seed=4))
    d.U_hat1[...] = d.U_hat
    tdt = torch.float64 if dtype == "float64" else torch.float32
    doms = [SlabDomain(n, nu=1e-3, dt=1e-3, method=method, les=les, Cs=0.17, dtype=tdt, nranks=P, rank=r,
                       exchange=lambda out, inp: None) for r in range(P)]
    for s in doms:
        s.set_state(d.U_hat)
    step = emulated_exchange(doms)
    ref_step = RK3_method.solveForNextTimestep if method == "RK3" else RK4_method.solveForNextTimestep
    for _ in range(3):
        umax_ref = float(d.U.max())
        step()
        ref_step(d)
    for s in doms:
        s.check()
    d._plan.check()
    got = torch.cat([s.local() for s in doms], dim=2)
    assert _rel(got, d.U_hat) < tol
    assert doms[0].u_max == pytest.approx(umax_ref, rel=10 * tol)
    del doms, d
    torch.cuda.empty_cache()


def test_slab_plan_refuses_whole_grid_calls():
    from sles import _native as nat
    sd = SlabDomain(64, nu=1e-3, dt=1e-3, method="RK3", les="Smagorinsky", dtype=torch.float64, nranks=2, rank=1,
                    exchange=lambda o, i: None)
    du = torch.zeros_like(sd.U_hat)
    with pytest.raises(nat.SlesError) as e:
        sd.plan.rhs(sd.U_hat, du)
    assert e.value.status == 7  # SLES_ERR_STATE
