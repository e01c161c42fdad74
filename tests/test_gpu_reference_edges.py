"""The drop-in surface around the fused steppers, against the reference's own
records (float64):

* the driver loop ``SM_solver.spectralMethodSolver`` with its adaptive dt, on
  the host and with the time-step logic on the GPU (``device_dt=True``),
  against the reference's own run of src/SM_solver.py:18-83 (steps taken,
  every dt of the host loop, the final dt and U_hat, the Ek_plot_data.csv
  columns and values);
* the operator helpers ``math_formula.velocity_gradient`` (the C-ABI entry
  point ``sles_velocity_gradient``), ``smagorinsky/vreman.calculate_nuR`` and
  ``math_formula.residue_stress`` against the reference's a_ij, nuR and
  temp_I (src/math_formula.py:27-127, src/smagorinsky.py:24-47,
  src/vreman.py:30-123);
* the diagnostics ``U_square``, ``dissipation_rate`` (src/RK4_method.py:77-101)
  and ``reference_binned_spectrum`` (calculate_Ek, src/SM_solver.py:154-192)
  against the reference's values, and ``sles_diag``'s compensated E, eps and
  shell spectrum against the oracle.

Tolerances: 1e-11 relative for fields and spectra after many steps, 1e-12 for
single operators and reductions; step counts and CSV column labels exact.
"""
import json
import os

import numpy as np
import pytest
import torch

import sles.SM_solver as smod
from conftest import GOLDEN, solver_cases
from oracle import spectral_oracle as so
from sles import diagnostics, math_formula, smagorinsky, vreman
from sles.initial import initial_velocity, initial_vorticity
from sles.initialize_domain import InitializeDomain

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def _load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return z, json.loads(str(z["meta"]))


def _solver_domain(z, meta):
    kw = {k: meta[k] for k in ("No_of_gridpoint", "dimension", "nu", "final_time", "method", "CFL")}
    for k in ("LES_ON", "LES_model", "Cs"):
        if k in meta:
            kw[k] = meta[k]
    d = InitializeDomain(**kw, dtype="float64")
    if "omega0" in z:
        initial_vorticity(d, z["omega0"])
    else:
        initial_velocity(d, *z["u0"])
    return d


def _check_csv(z):
    import pandas as pd
    csv = pd.read_csv("Ek_plot_data.csv")
    assert list(csv.columns) == json.loads(str(z["ek_columns"]))
    got = csv.to_numpy(dtype=float)
    ref = z["ek_values"]
    assert got.shape == ref.shape
    assert rel(got, ref) < 1e-11


@pytest.mark.parametrize("name", solver_cases())
def test_driver_loop_host_matches_reference(name, tmp_path, monkeypatch):
    z, meta = _load(name)
    d = _solver_domain(z, meta)
    dts = []
    orig = smod.compute_dt

    def rec(U, u_max, nu, comm=None, dx=1.0, CFL=0.5):
        dt = orig(U, u_max, nu, comm, dx=dx, CFL=CFL)
        dts.append(dt)
        return dt

    monkeypatch.setattr(smod, "compute_dt", rec)
    monkeypatch.chdir(tmp_path)
    steps = smod.spectralMethodSolver(d, file_out_time=0.0, No_Ek_plot=meta["No_Ek_plot"], verbose=False)
    assert steps == meta["steps"]
    np.testing.assert_allclose(dts, z["dt_seq"], rtol=1e-11)
    assert d.dt == pytest.approx(meta["dt_final"], rel=1e-11)
    assert rel(d.U_hat.cpu().numpy(), z["U_hat_final"]) < 1e-11
    _check_csv(z)


@pytest.mark.parametrize("name", solver_cases())
def test_driver_loop_device_dt_matches_reference(name, tmp_path, monkeypatch):
    z, meta = _load(name)
    d = _solver_domain(z, meta)
    monkeypatch.chdir(tmp_path)
    steps = smod.spectralMethodSolver(d, file_out_time=0.0, No_Ek_plot=meta["No_Ek_plot"], verbose=False,
                                      device_dt=True)
    assert steps == meta["steps"]
    assert d.dt == pytest.approx(meta["dt_final"], rel=1e-11)
    assert rel(d.U_hat.cpu().numpy(), z["U_hat_final"]) < 1e-11
    _check_csv(z)


@pytest.mark.parametrize("model", ["Smagorinsky", "vreman"])
def test_operator_helpers_match_reference(model):
    z = np.load(os.path.join(GOLDEN, "ops16.npz"))
    key = "noise_%s_" % model[0]
    d = InitializeDomain(No_of_gridpoint=64, dimension=3, nu=1e-2, time_stepSize=1e-3, method="RK4",
                         LES_ON=1, LES_model=model, Cs=0.17, dtype="float64")
    initial_velocity(d, *z[key + "u"])
    math_formula.velocity_gradient(d)  # sles_velocity_gradient through the plan
    A = np.array([[getattr(d, "a%d%d" % (i + 1, j + 1)).cpu().numpy() for j in range(3)] for i in range(3)])
    assert rel(A, z[key + "grad"]) < 1e-12
    (smagorinsky if model[0] == "S" else vreman).calculate_nuR(d)
    assert rel(d.nuR.cpu().numpy(), z[key + "nuR"]) < 1e-12
    T = math_formula.residue_stress(d)
    assert rel(T.cpu().numpy(), z[key + "temp_I"]) < 1e-12


def test_velocity_gradient_entry_point_on_band_limited_field():
    """sles_velocity_gradient (input slot reused as scratch by its c2r) on the
    seeded spectrum field: a_ij against the oracle's irfftn(i K_i U_hat_j)."""
    n = 32
    u = so.random_spectrum_velocity(n, k0=4.0, u0=1.0, seed=5)
    d = InitializeDomain(No_of_gridpoint=4 * n, dimension=3, nu=1e-3, method="RK4", LES_ON=1,
                         LES_model="Smagorinsky", Cs=0.17, dtype="float64")
    initial_velocity(d, *u)
    g = torch.empty((9, n, n, n), dtype=torch.float64, device=d.device)
    d._plan.velocity_gradient(d._s_uhat, g)
    o = so.OracleDomain(n, 3, nu=1e-3, les_model="Smagorinsky", Cs=0.17)
    so.initial_velocity(o, *u)
    A = so.velocity_gradient(o, o.U_hat)
    assert rel(g.cpu().numpy().reshape(3, 3, n, n, n), A) < 1e-12
    # the state is untouched by the call
    assert rel(d.U_hat.cpu().numpy(), o.U_hat) < 1e-13


def test_diagnostics_match_reference():
    z = np.load(os.path.join(GOLDEN, "diag16.npz"))
    for tag in ("rand16", "noise16", "vort32"):
        meta = json.loads(str(z[tag + "_meta"]))
        d = InitializeDomain(No_of_gridpoint=meta["N"], dimension=meta["dimension"], nu=meta["nu"],
                             method="RK4", dtype="float64")
        if tag + "_omega0" in z:
            initial_vorticity(d, z[tag + "_omega0"])
        else:
            initial_velocity(d, *z[tag + "_u0"])
        assert diagnostics.U_square(d) == pytest.approx(float(z[tag + "_U_square"]), rel=1e-12)
        assert diagnostics.dissipation_rate(d) == pytest.approx(float(z[tag + "_dissipation_rate"]), rel=1e-12)
        tk, tE = diagnostics.reference_binned_spectrum(d)
        np.testing.assert_allclose(tk, z[tag + "_temp_k"], rtol=1e-13)
        # bins beyond the field's band hold round-off-level energy: an absolute floor
        np.testing.assert_allclose(tE, z[tag + "_temp_Ek"], rtol=1e-12, atol=1e-14 * np.max(z[tag + "_temp_Ek"]))


@pytest.mark.parametrize("dim,n", [(3, 16), (3, 32), (2, 64)])
def test_device_diag_matches_oracle(dim, n):
    """sles_diag: float64 compensated E, eps, signed max of u and the
    integer-shell spectrum, against the oracle's NumPy sums."""
    rng = np.random.default_rng(7 + n)
    f = [rng.standard_normal((n,) * dim) for _ in range(dim)]
    d = InitializeDomain(No_of_gridpoint=n, dimension=dim, nu=2e-3, method="RK4", dtype="float64")
    initial_velocity(d, *f)
    o = so.OracleDomain(n, dim, nu=2e-3)
    so.initial_velocity(o, *f)
    E, eps, umax, nonfinite, spec = diagnostics.diag(d, with_max=True, nshell=int(0.5 * n * np.sqrt(dim)) + 2)
    assert not nonfinite
    assert E == pytest.approx(so.energy(o), rel=1e-13)
    assert eps == pytest.approx(so.dissipation(o), rel=1e-13)
    assert umax == np.max(np.array(f))
    ref = so.shell_spectrum(o)
    m = min(ref.size, spec.size)
    assert rel(spec[:m], ref[:m]) < 1e-13
    assert np.all(ref[m:] == 0) and np.all(spec[m:] == 0)
