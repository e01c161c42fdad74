"""Failure detection without a GPU fault: a kernel whose wait runs out (an
mbarrier that nothing arrives at) reports SLES_ERR_TIMEOUT through the plan's
error word, and the context stays usable."""
import ctypes

import pytest
import torch

from sles import RK3_method
from sles import _native as nat
from sles.initial import initial_velocity
from sles.initialize_domain import InitializeDomain
from sles.synthetic import random_spectrum_velocity

pytestmark = pytest.mark.gpu


def test_wait_timeout_is_reported_and_context_survives():
    d = InitializeDomain(nu=1e-3, dimension=3, time_stepSize=1e-3, No_of_gridpoint=4 * 32, method="RK3", LES_ON=1,
                         LES_model="Smagorinsky", Cs=0.17, dtype="float32")
    initial_velocity(d, *random_spectrum_velocity(32, 4.0, 1.0, seed=1))
    assert d._plan.check() == 0
    d._plan.selftest_wait_timeout()
    with pytest.raises(nat.SlesError) as e:
        d._plan.check()
    assert e.value.status == 5  # SLES_ERR_TIMEOUT
    assert d._plan.check() == 0  # the word was cleared
    for _ in range(2):
        RK3_method.solveForNextTimestep(d)
    assert d._plan.check() == 0
    assert bool(torch.isfinite(d.U_hat.abs()).all())


def test_adjoint_workspace_timeout_is_reported():
    """The reverse passes report bounded-wait timeouts in the adjoint
    workspace's own header word, read by sles_adjoint_check."""
    from sles.adjoint import RK4Rollout
    ro = RK4Rollout(32, 1e-3, 1e-3, les="Smagorinsky", Cs=0.17, dtype=torch.float32)
    assert ro.plan.adjoint_check(ro._ws) == 0
    L = nat.load_library()
    assert L.sles_selftest_wait_timeout_word(ctypes.c_void_p(ro._ws), nat.stream_handle(ro.device)) == 0
    with pytest.raises(nat.SlesError) as e:
        ro.plan.adjoint_check(ro._ws)
    assert e.value.status == 5  # SLES_ERR_TIMEOUT
    assert ro.plan.adjoint_check(ro._ws) == 0  # cleared
    assert ro.plan.check() == 0  # the forward plan's word is separate
