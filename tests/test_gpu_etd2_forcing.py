"""Corrected ETD2 (Cox-Matthews) with linear forcing, against the oracle.

The reference's ETD2 forcing branch cannot run (src/ETD2_method.py:47-50
reads domain.epsilon, which is never set), so this case has no golden
vectors: the fused float64 path is checked against the oracle's restatement,
which treats the forcing f U_hat (k != 0) explicitly, inside the term the
exponential integrator weights.  Bar: relative L2 error of U_hat below 1e-11
after every step.
"""
import numpy as np
import pytest

from oracle import spectral_oracle as so
from sles import ETD2_method
from sles.initial import initial_velocity
from sles.initialize_domain import InitializeDomain

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("les", [None, "Smagorinsky"])
def test_corrected_etd2_with_forcing_matches_oracle(les):
    n, nu, dt, f, cs = 32, 4e-3, 4e-3, 0.05, 0.17
    o = so.OracleDomain(n, 3, nu=nu, dt=dt, les_model=les, Cs=cs, method="ETD2", forcing=f, parity=False)
    d = InitializeDomain(nu=nu, dimension=3, time_stepSize=dt, No_of_gridpoint=(4 if les else 1) * n,
                         method="ETD2", LES_ON=1 if les else 0, LES_model=les, Cs=cs, forcing=f,
                         dtype="float64", parity_mode=False)
    u, v, w = so.random_spectrum_velocity(n, 3.0, 1.0, seed=8)
    so.initial_velocity(o, u, v, w)
    initial_velocity(d, u, v, w)
    o.U_hat1 = o.U_hat.copy()
    d.U_hat1[...] = d.U_hat
    for _ in range(5):
        so.step(o)
        o.U_hat1 = o.U_hat.copy()
        ETD2_method.solveForNextTimestep(d)
        got = d.U_hat.cpu().numpy()
        err = np.linalg.norm(got - o.U_hat) / np.linalg.norm(o.U_hat)
        assert err < 1e-11


def test_reference_etd2_forcing_error_is_kept():
    d = InitializeDomain(nu=4e-3, dimension=3, time_stepSize=4e-3, No_of_gridpoint=16, method="ETD2", forcing=0.05,
                         dtype="float64")
    u, v, w = so.random_spectrum_velocity(16, 3.0, 1.0, seed=8)
    initial_velocity(d, u, v, w)
    d.U_hat1[...] = d.U_hat
    ETD2_method.solveForNextTimestep(d)       # the RK4 bootstrap step runs
    with pytest.raises(AttributeError):
        ETD2_method.solveForNextTimestep(d)   # as src/ETD2_method.py:47-50
