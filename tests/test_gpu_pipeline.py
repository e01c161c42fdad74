"""HostStepper: host-resident states advanced with overlapped copies give the
same results as copying in, stepping and copying out one at a time."""
import pytest
import torch

from sles import ETD2_method, RK3_method, RK4_method
from sles.initial import initial_velocity
from sles.initialize_domain import InitializeDomain
from sles.pipeline import HostStepper
from sles.synthetic import random_spectrum_velocity

pytestmark = pytest.mark.gpu
STEP = {"RK3": RK3_method.solveForNextTimestep, "RK4": RK4_method.solveForNextTimestep,
        "ETD2": ETD2_method.solveForNextTimestep}


def _dom(method):
    d = InitializeDomain(nu=1e-3, dimension=3, time_stepSize=2e-3, No_of_gridpoint=4 * 48, method=method, LES_ON=1,
                         LES_model="Smagorinsky", Cs=0.17, dtype="float32", parity_mode=(method != "ETD2"))
    initial_velocity(d, *random_spectrum_velocity(48, 4.0, 1.0, seed=1))
    d.U_hat1[...] = d.U_hat
    return d


@pytest.mark.parametrize("method", ["RK3", "RK4", "ETD2"])
def test_host_stepper_matches_one_at_a_time(method):
    d = _dom(method)
    states = []
    for s in range(4):
        u, v, w = random_spectrum_velocity(48, 4.0, 1.0, seed=10 + s)
        states.append(torch.fft.rfftn(torch.stack([u, v, w]), dim=(1, 2, 3)).to(torch.complex64).cpu().pin_memory())
    outs = [torch.empty_like(x).pin_memory() for x in states]
    hs = HostStepper(d, steps=3)
    hs.run(states, outs)
    hs.synchronize()
    for x, y in zip(states, outs):
        r = _dom(method)
        r.U_hat[...] = x.cuda()
        r.U_hat1[...] = r.U_hat
        r._mark_stepped()
        for _ in range(3):
            STEP[method](r)
        ref = r.U_hat.cpu()
        assert torch.equal(y, ref)
    assert hs.bytes_in == hs.bytes_out == sum(x.numel() * x.element_size() for x in states)
