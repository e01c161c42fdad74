"""The CPU oracle against golden vectors produced by the reference's own code.

The fixtures in ``tests/golden`` were written by ``tests/golden/make_golden.py``,
which runs the reference's unmodified ``src/`` under a single-rank shim.  These
tests pin the oracle (``oracle/spectral_oracle.py``) to them, so that every
GPU parity test that compares against the oracle is transitively anchored on
the reference.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, solver_cases, step_cases
from oracle import spectral_oracle as so

CASES = step_cases()


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return z, json.loads(str(z["meta"]))


def make_domain(meta):
    return so.OracleDomain.from_reference_args(
        meta["No_of_gridpoint"], dimension=meta["dimension"], nu=meta["nu"],
        time_stepSize=meta["time_stepSize"], LES_ON=meta.get("LES_ON", 0),
        LES_model=meta.get("LES_model"), Cs=meta.get("Cs", 0.14),
        method=meta["method"], forcing=meta.get("forcing", 0.0), parity=True)


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_steps(name):
    z, meta = load(name)
    d = make_domain(meta)
    assert d.N == meta["N"]
    if "omega0" in z:
        so.initial_vorticity(d, z["omega0"])
    else:
        so.initial_velocity(d, *z["u0"])
    if "U_hat_init" in z:
        assert rel(d.U_hat, z["U_hat_init"]) < 1e-14
    d.U_hat1 = d.U_hat.copy()
    for s in range(meta["steps"]):
        so.step(d)
        err = rel(d.U_hat, z["U_hat_%d" % (s + 1)])
        assert err < 1e-12, (name, s + 1, err)
    if "U_final" in z:
        assert rel(d.U, z["U_final"]) < 1e-12
        assert rel(d.curl, z["curl_final"]) < 1e-12


@pytest.mark.parametrize("model", ["S", "v"])
def test_oracle_operators(model):
    z = np.load(os.path.join(GOLDEN, "ops16.npz"))
    key = "noise_%s_" % model
    d = so.OracleDomain(16, 3, nu=1e-2, dt=1e-3,
                        les_model="Smagorinsky" if model == "S" else "vreman", Cs=0.17)
    so.initial_velocity(d, *z[key + "u"])
    assert rel(d.U_hat, z[key + "U_hat"]) < 1e-14
    assert rel(d.curl, z[key + "curl"]) < 1e-13
    A = so.velocity_gradient(d, d.U_hat)
    assert rel(A, z[key + "grad"]) < 1e-13
    nu = so.nuR_smagorinsky(d, A) if model == "S" else so.nuR_vreman(d, A)
    assert rel(nu, z[key + "nuR"]) < 1e-13
    T = so.residue_stress(d, A, nu)
    assert rel(T, z[key + "temp_I"]) < 1e-13
    dU0 = so.compute_rhs(d, 0).copy()
    assert rel(dU0, z[key + "dU_rk0"]) < 1e-13
    dU1 = so.compute_rhs(d, 1).copy()
    assert rel(dU1, z[key + "dU_rk1"]) < 1e-13


def test_taylor_green_early_decay():
    """E(t) = 1/8 exp(-6 nu t) + O(t^2) for the 3D Taylor-Green vortex."""
    d = so.OracleDomain(16, 3, nu=1 / 1600, dt=0.01, method="RK4")
    so.initial_velocity(d, *so.taylor_green(16))
    d.U_hat1 = d.U_hat.copy()
    assert abs(so.energy(d) - 0.125) < 1e-14
    for _ in range(10):
        so.step(d)
    exact = 0.125 * np.exp(-6 * d.nu * 0.1)
    assert abs(so.energy(d) - exact) / exact < 1e-6


def test_random_spectrum_is_solenoidal_and_scaled():
    n = 32
    u = np.array(so.random_spectrum_velocity(n, k0=4.0, u0=1.0, seed=3))
    d = so.OracleDomain(n, 3)
    so.initial_velocity(d, *u)
    div = np.sum(d.K * d.U_hat, 0)
    assert np.max(np.abs(div)) < 1e-9 * np.max(np.abs(d.U_hat))
    # energy of the truncated model spectrum on the resolved shells
    E = so.shell_spectrum(d)
    k = np.arange(E.size, dtype=float)
    target = so._model_spectrum(k, 4.0, 1.0)
    kc = int(2.0 / 3.0 * (n // 2 + 1))
    np.testing.assert_allclose(E[1:kc - 3], target[1:kc - 3], rtol=1e-10)


def test_etd2_corrected_coefficients_limit():
    K2 = np.array([0, 1, 2, 3, 10**6])
    E, c1, c0 = so.etd2_coefficients(K2, nu=1e-4, dt=1e-3, parity=False)
    assert c1[0] == pytest.approx(1.5e-3) and c0[0] == pytest.approx(-0.5e-3)
    # series and closed forms agree where both are accurate
    z = 1e-4 * 1e-3 * 10**6
    c1x = 1e-3 * ((1 - z) * np.exp(-z) - 1 + 2 * z) / z**2
    assert c1[-1] == pytest.approx(c1x, rel=1e-12)


def _oracle_from_solver_meta(meta):
    return so.OracleDomain.from_reference_args(
        meta["No_of_gridpoint"], dimension=meta["dimension"], nu=meta["nu"], LES_ON=meta.get("LES_ON", 0),
        LES_model=meta.get("LES_model"), Cs=meta.get("Cs", 0.14), method=meta["method"], parity=True)


@pytest.mark.parametrize("name", solver_cases())
def test_oracle_driver_loop_matches_reference(name):
    """The oracle's restatement of spectralMethodSolver (adaptive dt, E(k)
    snapshots) against the reference's own run of it."""
    z, meta = load(name)
    d = _oracle_from_solver_meta(meta)
    if "omega0" in z:
        so.initial_vorticity(d, z["omega0"])
    else:
        so.initial_velocity(d, *z["u0"])
    steps, dts, umaxs, snaps = so.solver_loop(d, meta["final_time"], CFL=meta["CFL"], No_Ek_plot=meta["No_Ek_plot"])
    assert steps == meta["steps"]
    np.testing.assert_allclose(dts, z["dt_seq"], rtol=1e-12)
    np.testing.assert_allclose(umaxs, z["umax_seq"], rtol=1e-12)
    assert rel(d.U_hat, z["U_hat_final"]) < 1e-11
    cols = json.loads(str(z["ek_columns"]))
    assert cols == [c for t, _, _ in snaps for c in ("k-%g" % t, "Ek-%g" % t)]
    vals = np.concatenate([np.stack([tk, tE], 1) for _, tk, tE in snaps], 1)
    np.testing.assert_allclose(vals, z["ek_values"], rtol=1e-11, atol=0)


def test_oracle_diagnostics_match_reference():
    z = np.load(os.path.join(GOLDEN, "diag16.npz"))
    for tag in ("rand16", "noise16", "vort32"):
        meta = json.loads(str(z[tag + "_meta"]))
        d = so.OracleDomain(meta["N"], meta["dimension"], nu=meta["nu"])
        if tag + "_omega0" in z:
            so.initial_vorticity(d, z[tag + "_omega0"])
        else:
            so.initial_velocity(d, *z[tag + "_u0"])
        assert so.U_square(d) == pytest.approx(float(z[tag + "_U_square"]), rel=1e-13)
        assert so.dissipation_rate(d) == pytest.approx(float(z[tag + "_dissipation_rate"]), rel=1e-12)
        tk, tE = so.reference_binned_spectrum(d)
        np.testing.assert_allclose(tk, z[tag + "_temp_k"], rtol=1e-14)
        np.testing.assert_allclose(tE, z[tag + "_temp_Ek"], rtol=1e-12)
