"""Fused CUDA path (float64) against the reference's own outputs.

Every golden fixture (written by the reference solver under a single-rank
shim, tests/golden/make_golden.py) is replayed through the drop-in API:
InitializeDomain + initial_velocity/initial_vorticity + solveForNextTimestep.
Bar: relative L2 error of U_hat below 1e-11 after every step.
"""
import json
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, step_cases
from sles import ETD2_method, RK3_method, RK4_method
from sles.initial import initial_velocity, initial_vorticity
from sles.initialize_domain import InitializeDomain

pytestmark = pytest.mark.gpu
CASES = step_cases()
STEP = {"RK4": RK4_method, "RK3": RK3_method, "ETD2": ETD2_method}


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def make(meta, dtype="float64"):
    kw = {k: meta[k] for k in ("No_of_gridpoint", "dimension", "nu", "time_stepSize", "method") if k in meta}
    for k in ("LES_ON", "LES_model", "Cs", "forcing"):
        if k in meta:
            kw[k] = meta[k]
    return InitializeDomain(**kw, dtype=dtype)


@pytest.mark.parametrize("name", CASES)
def test_fused_float64_matches_reference(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    d = make(meta)
    if "omega0" in z:
        initial_vorticity(d, z["omega0"])
    else:
        initial_velocity(d, *z["u0"])
    if "U_hat_init" in z:
        assert rel(d.U_hat.cpu().numpy(), z["U_hat_init"]) < 1e-13
    d.U_hat1[...] = d.U_hat
    for s in range(meta["steps"]):
        STEP[meta["method"]].solveForNextTimestep(d)
        err = rel(d.U_hat.cpu().numpy(), z["U_hat_%d" % (s + 1)])
        assert err < 1e-11, (name, s + 1, err)
    if "U_final" in z:
        assert rel(d.U.cpu().numpy(), z["U_final"]) < 1e-11
        assert rel(d.curl.cpu().numpy(), z["curl_final"]) < 1e-11


@pytest.mark.parametrize("model", ["Smagorinsky", "vreman"])
def test_compute_rhs_matches_reference(model):
    z = np.load(os.path.join(GOLDEN, "ops16.npz"))
    key = "noise_%s_" % model[0]
    d = InitializeDomain(No_of_gridpoint=64, dimension=3, nu=1e-2, time_stepSize=1e-3, method="RK4",
                         LES_ON=1, LES_model=model, Cs=0.17, dtype="float64")
    initial_velocity(d, *z[key + "u"])
    assert rel(d.curl.cpu().numpy(), z[key + "curl"]) < 1e-13
    dU = RK4_method.computeRHS(d, None, 0).cpu().numpy()
    assert rel(dU, z[key + "dU_rk0"]) < 1e-12
    dU = RK4_method.computeRHS(d, None, 1).cpu().numpy()
    assert rel(dU, z[key + "dU_rk1"]) < 1e-12
