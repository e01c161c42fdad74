"""The plain torch path (comparison path and autograd reference) against the
oracle on CPU: RHS and steps at small sizes to 1e-12."""
import numpy as np
import pytest
import torch

from oracle import spectral_oracle as so
from sles.plain_torch import PlainSolver

CASES = [
    dict(n=16, dim=3, les=None, method="RK4", parity=True),
    dict(n=16, dim=3, les="Smagorinsky", method="RK4", parity=True),
    dict(n=16, dim=3, les="vreman", method="RK3", parity=True),
    dict(n=24, dim=3, les="Smagorinsky", method="RK3", parity=False),
    dict(n=16, dim=3, les="Smagorinsky", method="ETD2", parity=False),
    dict(n=32, dim=2, les=None, method="RK4", parity=True),
]


def _pair(c):
    o = so.OracleDomain(c["n"], c["dim"], nu=2e-3, dt=2e-3, les_model=c["les"], Cs=0.17, method=c["method"],
                        parity=c["parity"])
    p = PlainSolver(c["n"], c["dim"], nu=2e-3, dt=2e-3, les=c["les"], Cs=0.17, method=c["method"],
                    parity=c["parity"], device="cpu")
    if c["dim"] == 3:
        so.initial_velocity(o, *so.random_spectrum_velocity(c["n"], 3.0, 1.0, seed=5))
    else:
        so.initial_vorticity(o, so.gaussian_vorticity_2d(c["n"], seed=5, kp=4.0))
    o.U_hat1 = o.U_hat.copy()
    return o, p


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("c", CASES, ids=lambda c: "%s%d_%s_%s_%s" % ("3d" if c["dim"] == 3 else "2d", c["n"],
                                                                      c["les"], c["method"], c["parity"]))
def test_plain_torch_matches_oracle(c):
    o, p = _pair(c)
    Uh = torch.as_tensor(o.U_hat.copy())
    if c["method"] != "ETD2":
        r = p.rhs(Uh)
        ro = so.compute_rhs(o, 1)
        assert rel(r.numpy(), ro) < 1e-12
    for _ in range(3):
        Uh = p.step(Uh)
        so.step(o)
        o.U_hat1 = o.U_hat.copy()
    assert rel(Uh.numpy(), o.U_hat) < 1e-12


def test_shell_spectrum_matches_oracle():
    o, p = _pair(CASES[1])
    e = p.shell_spectrum(torch.as_tensor(o.U_hat)).numpy()
    eo = so.shell_spectrum(o)
    assert np.allclose(e, eo[: len(e)], rtol=1e-12, atol=0)
