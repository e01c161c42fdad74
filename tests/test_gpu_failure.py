"""Failure detection without a GPU fault: a kernel whose wait runs out (an
mbarrier that nothing arrives at) reports SLES_ERR_TIMEOUT through the plan's
error word, and the context stays usable."""
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
