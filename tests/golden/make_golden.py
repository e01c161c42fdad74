"""Generate the golden fixtures in this folder from the reference solver itself.

Runs the reference's own, unmodified ``src/`` modules (a-k-sangwan/spectral-LES)
from a checkout of the reference under a single-rank shim and stores their
outputs as ``.npz`` files.  The shim only replaces the third-party layer the reference
imports but that is not installed here:

* ``mpi4py.MPI``: COMM_WORLD of size 1, Allreduce copies send -> recv;
* ``mpi4py_fft.PFFT``: forward(normalize=False) = numpy.fft.rfftn,
  backward(normalize=True) = numpy.fft.irfftn (the PFFT conventions at the
  reference's call sites, src/math_formula.py:7-24); ``newDistArray`` = zeros;
* ``HDF5File``, ``mpi4py_fft.io.generate_xdmf`` and ``matplotlib.pyplot``:
  inert stubs (output and plotting are not on the measured path).

The integrators are driven with a fixed dt (``solveForNextTimestep`` called
directly after ``U_hat1[:] = U_hat``, as src/SM_solver.py:33 does), because
``spectralMethodSolver`` overrides dt (src/SM_solver.py:22-24, 61-63).
The driver loop itself is recorded separately (``solver_*.npz``): the
reference's ``spectralMethodSolver`` runs with its adaptive dt in a scratch
directory, and the fixture keeps every dt and u_max it computed (its own
``compute_dt``, wrapped to record them), the number of steps, the final
U_hat and the ``Ek_plot_data.csv`` it wrote.  ``diag16.npz`` keeps the
reference's ``U_square``, ``dissipation_rate`` (src/RK4_method.py:77-101) and
``calculate_Ek`` bins (src/SM_solver.py:154-192) on seeded fields.
Initial fields come from the oracle's seeded generators so both sides see
identical inputs; they are stored in the fixtures too.

Usage (the path of a reference checkout is required):
    python tests/golden/make_golden.py --reference <path> [--only steps,ops,solver,diag]
or set SLES_REFERENCE=<path>.
"""
from __future__ import annotations

import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("SLES_REFERENCE")


def install_shim():
    """Register fake mpi4py / mpi4py_fft / matplotlib modules in sys.modules."""
    mpi = types.ModuleType("mpi4py.MPI")

    class _Req:
        def wait(self):
            return None

    class _Comm:
        rank = 0

        def Get_size(self):
            return 1

        def Get_rank(self):
            return 0

        def Allreduce(self, send, recv, op=None):
            s = send[0] if isinstance(send, (list, tuple)) else send
            r = recv[0] if isinstance(recv, (list, tuple)) else recv
            np.asarray(r).reshape(-1)[0] = np.asarray(s).reshape(-1)[0]

        def Isend(self, *a, **k):
            return _Req()

        def Irecv(self, *a, **k):
            return _Req()

    mpi.COMM_WORLD = _Comm()
    mpi.DOUBLE, mpi.FLOAT, mpi.MAX, mpi.SUM = "d", "f", "max", "sum"
    pkg = types.ModuleType("mpi4py")
    pkg.MPI = mpi
    sys.modules["mpi4py"] = pkg
    sys.modules["mpi4py.MPI"] = mpi

    fftmod = types.ModuleType("mpi4py_fft")

    class PFFT:
        def __init__(self, comm, shape, axes=None, dtype=float, grid=None):
            self.shape = tuple(int(s) for s in shape)
            self.axes = tuple(range(len(self.shape)))
            self.ntot = float(np.prod(self.shape))

        def forward(self, a, out=None, normalize=False):
            r = np.fft.rfftn(np.asarray(a), axes=self.axes)
            if normalize:
                r = r / self.ntot
            if out is not None:
                out[...] = r
                return out
            return r

        def backward(self, a, out=None, normalize=True):
            r = np.fft.irfftn(np.asarray(a), s=self.shape, axes=self.axes)
            if not normalize:
                r = r * self.ntot
            if out is not None:
                out[...] = r
                return out
            return r

    def newDistArray(fft, forward_output=True):
        if forward_output:
            shp = fft.shape[:-1] + (fft.shape[-1] // 2 + 1,)
            return np.zeros(shp, dtype=complex)
        return np.zeros(fft.shape)

    class HDF5File:
        def __init__(self, *a, **k):
            pass

        def write(self, *a, **k):
            pass

    fftmod.PFFT, fftmod.newDistArray, fftmod.HDF5File = PFFT, newDistArray, HDF5File
    io = types.ModuleType("mpi4py_fft.io")
    io.generate_xdmf = lambda *a, **k: None
    fftmod.io = io
    sys.modules["mpi4py_fft"] = fftmod
    sys.modules["mpi4py_fft.io"] = io

    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")

    class _Ax:
        # figure/axes stand-in: every method returns another stand-in, and the
        # position box read by save_Ek_plot (src/SM_solver.py:234-235) exists
        x0 = y0 = width = height = 0.0

        def __getattr__(self, name):
            return lambda *a, **k: _Ax()

    plt.subplots = lambda *a, **k: (_Ax(), _Ax())
    plt.rcParams = {}
    plt.close = lambda *a, **k: None
    mpl.pyplot = plt
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt


def import_reference():
    if not REF or not os.path.isdir(os.path.join(REF, "src")):
        raise SystemExit("make_golden.py needs the reference checkout: --reference <path> or SLES_REFERENCE")
    install_shim()
    if REF not in sys.path:
        sys.path.insert(0, REF)
    import importlib
    mods = {}
    for name in ["initialize_domain", "initial", "math_formula", "smagorinsky",
                 "vreman", "RK4_method", "RK3_method", "ETD2_method", "SM_solver"]:
        mods[name] = importlib.import_module("src." + name)
    return mods


def _ic(kind, n, dim, seed, k0=4.0, mean=0.0):
    sys.path.insert(0, REPO)
    from oracle import spectral_oracle as so
    if kind == "tg":
        return so.taylor_green(n)
    if kind == "rand":
        return so.random_spectrum_velocity(n, k0=k0, u0=1.0, seed=seed)
    if kind == "noise":
        rng = np.random.default_rng(seed)
        return tuple(rng.standard_normal((n,) * dim) for _ in range(dim))
    if kind == "vort":
        return (so.gaussian_vorticity_2d(n, seed=seed) + mean,)
    raise ValueError(kind)


CASES = [
    # name, reference kwargs, ic, steps
    ("tg16_rk4", dict(No_of_gridpoint=16, dimension=3, nu=1 / 1600, time_stepSize=0.01,
                      method="RK4", LES_ON=0), ("tg", 0), 3),
    ("rand16_rk3_smag", dict(No_of_gridpoint=64, dimension=3, nu=1e-3, time_stepSize=5e-3,
                             method="RK3", LES_ON=1, LES_model="Smagorinsky", Cs=0.17),
     ("rand", 1), 3),
    ("rand16_rk4_vreman", dict(No_of_gridpoint=64, dimension=3, nu=1e-3, time_stepSize=5e-3,
                               method="RK4", LES_ON=1, LES_model="vreman", Cs=0.16733),
     ("rand", 2), 2),
    ("rand16_etd2", dict(No_of_gridpoint=16, dimension=3, nu=1e-2, time_stepSize=5e-3,
                         method="ETD2", LES_ON=0), ("rand", 3), 3),
    ("rand16_etd2_smag", dict(No_of_gridpoint=64, dimension=3, nu=1e-2, time_stepSize=5e-3,
                              method="ETD2", LES_ON=1, LES_model="Smagorinsky", Cs=0.17),
     ("rand", 4), 3),
    ("rand16_rk4_forcing", dict(No_of_gridpoint=16, dimension=3, nu=1e-2, time_stepSize=5e-3,
                                method="RK4", LES_ON=0, forcing=0.1), ("rand", 5), 2),
    ("rand24_rk4_smag", dict(No_of_gridpoint=96, dimension=3, nu=1e-3, time_stepSize=5e-3,
                             method="RK4", LES_ON=1, LES_model="Smagorinsky", Cs=0.15),
     ("rand", 6), 2),
    ("noise16_rk4_smag", dict(No_of_gridpoint=64, dimension=3, nu=1e-2, time_stepSize=1e-3,
                              method="RK4", LES_ON=1, LES_model="Smagorinsky", Cs=0.17),
     ("noise", 7), 2),
    ("noise16_rk4_vreman", dict(No_of_gridpoint=64, dimension=3, nu=1e-2, time_stepSize=1e-3,
                                method="RK4", LES_ON=1, LES_model="vreman", Cs=0.17),
     ("noise", 8), 1),
    ("vort32_2d_rk4", dict(No_of_gridpoint=32, dimension=2, nu=1e-3, time_stepSize=5e-3,
                           method="RK4", LES_ON=0), ("vort", 9), 3),
    ("vort32_2d_rk4_smag", dict(No_of_gridpoint=128, dimension=2, nu=1e-3, time_stepSize=5e-3,
                                method="RK4", LES_ON=1, LES_model="Smagorinsky", Cs=0.17),
     ("vort", 10), 2),
    ("vort32_2d_rk3", dict(No_of_gridpoint=32, dimension=2, nu=1e-3, time_stepSize=5e-3,
                           method="RK3", LES_ON=0), ("vort", 11), 2),
    ("rand32_rk3_smag", dict(No_of_gridpoint=128, dimension=3, nu=1e-4, time_stepSize=1e-3,
                             method="RK3", LES_ON=1, LES_model="Smagorinsky", Cs=0.17),
     ("rand", 12), 1),
]


def run_case(ref, name, kw, ic, steps):
    D = ref["initialize_domain"].InitializeDomain
    d = D(**kw)
    kind, seed = ic
    if kind == "vort":
        (omega,) = _ic(kind, d.N, d.dim, seed, mean=0.25)
        ref["initial"].initial_vorticity(d, omega)
        fields = {"omega0": omega}
    else:
        f = _ic(kind, d.N, d.dim, seed)
        ref["initial"].initial_velocity(d, *f)
        fields = {"u0": np.array(f)}
    d.U_hat1[:] = d.U_hat[:]
    mod = {"RK4": "RK4_method", "RK3": "RK3_method", "ETD2": "ETD2_method"}[kw["method"]]
    stepper = ref[mod].solveForNextTimestep
    out = dict(fields)
    if d.dim == 2 or d.N <= 16:
        out["U_hat_init"] = np.array(d.U_hat)
    for s in range(steps):
        stepper(d)
        out["U_hat_%d" % (s + 1)] = np.array(d.U_hat).copy()
    if d.dim == 2 or kind == "tg":
        out["U_final"] = np.array(d.U)
        out["curl_final"] = np.array(d.curl)
    meta = dict(kw)
    meta.update(N=d.N, dim=d.dim, steps=steps, ic=kind, seed=seed)
    out["meta"] = np.array(json.dumps(meta))
    return out


def run_ops(ref):
    """Operator-level fixture on a noise field (all modes, Nyquist included)
    and a band-limited field: curl, gradients, nu_t, residue stress, dU."""
    D = ref["initialize_domain"].InitializeDomain
    mf = ref["math_formula"]
    out = {}
    for tag, kind, seed in (("noise", "noise", 21),):
        for model in ("Smagorinsky", "vreman"):
            d = D(No_of_gridpoint=64, dimension=3, nu=1e-2, time_stepSize=1e-3,
                  method="RK4", LES_ON=1, LES_model=model, Cs=0.17)
            f = _ic(kind, d.N, 3, seed)
            ref["initial"].initial_velocity(d, *f)
            key = "%s_%s_" % (tag, model[0])
            out[key + "u"] = np.array(f)
            out[key + "U_hat"] = np.array(d.U_hat)
            out[key + "curl"] = np.array(d.curl)
            mf.velocity_gradient(d)
            out[key + "grad"] = np.array([[d.a11, d.a12, d.a13], [d.a21, d.a22, d.a23],
                                          [d.a31, d.a32, d.a33]])
            if model[0] == "S":
                ref["smagorinsky"].calculate_nuR(d)
            else:
                ref["vreman"].calculate_nuR(d)
            out[key + "nuR"] = np.array(d.nuR)
            out[key + "temp_I"] = np.array(mf.residue_stress(d))
            dU = np.zeros_like(d.U_hat)
            out[key + "dU_rk0"] = np.array(ref["RK4_method"].computeRHS(d, dU, 0))
            dU = np.zeros_like(d.U_hat)
            out[key + "dU_rk1"] = np.array(ref["RK4_method"].computeRHS(d, dU, 1))
    out["meta"] = np.array(json.dumps(dict(N=16, No_of_gridpoint=64, nu=1e-2, Cs=0.17)))
    return out


SOLVER_CASES = [
    # name, reference kwargs (final_time included), ic, No_Ek_plot
    ("solver_rk3_smag16", dict(No_of_gridpoint=64, dimension=3, nu=1e-3, final_time=1.3, method="RK3",
                               LES_ON=1, LES_model="Smagorinsky", Cs=0.17, CFL=0.5), ("rand", 31), 5),
    ("solver_rk4_tg16", dict(No_of_gridpoint=16, dimension=3, nu=1 / 1600, final_time=2.5, method="RK4",
                             LES_ON=0, CFL=0.5), ("tg", 0), 4),
    ("solver_rk4_vort32_2d", dict(No_of_gridpoint=32, dimension=2, nu=1e-3, final_time=5.0, method="RK4",
                                  LES_ON=0, CFL=0.5), ("vort", 32), 3),
]


def run_solver(ref, name, kw, ic, n_ek):
    """The reference's spectralMethodSolver (src/SM_solver.py:18-83) with its
    adaptive dt, run in a scratch directory; records the dt / u_max sequence
    of its own compute_dt (wrapped), the steps taken, the final U_hat and
    the Ek_plot_data.csv it wrote."""
    import contextlib
    import io
    import tempfile

    import pandas as pd
    sm = ref["SM_solver"]
    D = ref["initialize_domain"].InitializeDomain
    d = D(**kw)
    kind, seed = ic
    out = {}
    if kind == "vort":
        (omega,) = _ic(kind, d.N, d.dim, seed, mean=0.0)
        ref["initial"].initial_vorticity(d, omega)
        out["omega0"] = omega
    else:
        f = _ic(kind, d.N, d.dim, seed)
        ref["initial"].initial_velocity(d, *f)
        out["u0"] = np.array(f)
    rec = {"dt": [], "umax": [], "steps": 0}
    orig_cd = sm.compute_dt
    step_mod = {"RK4": sm.RK4, "RK3": sm.RK3, "ETD2": sm.ETD2}[kw["method"]]
    orig_step = step_mod.solveForNextTimestep

    def compute_dt(U, u_max, nu, comm, dx, CFL=0.5):
        dt = orig_cd(U, u_max, nu, comm, dx=dx, CFL=CFL)
        rec["dt"].append(float(dt))
        rec["umax"].append(float(u_max))
        return dt

    def step(domain):
        rec["steps"] += 1
        return orig_step(domain)

    cwd = os.getcwd()
    sm.compute_dt, step_mod.solveForNextTimestep = compute_dt, step
    try:
        with tempfile.TemporaryDirectory() as tmp:
            os.chdir(tmp)
            with contextlib.redirect_stdout(io.StringIO()):
                sm.spectralMethodSolver(d, file_out_time=0.0, No_Ek_plot=n_ek)
            csv = pd.read_csv("Ek_plot_data.csv")
    finally:
        os.chdir(cwd)
        sm.compute_dt, step_mod.solveForNextTimestep = orig_cd, orig_step
    out["dt_seq"] = np.array(rec["dt"])
    out["umax_seq"] = np.array(rec["umax"])
    out["U_hat_final"] = np.array(d.U_hat)
    out["ek_columns"] = np.array(json.dumps(list(csv.columns)))
    out["ek_values"] = csv.to_numpy(dtype=float)
    # the loop's time: t = dt_0, then t += dt before each step (src/SM_solver.py:25, 51)
    t = rec["dt"][0] + sum(rec["dt"][:rec["steps"]])
    meta = dict(kw)
    meta.update(N=d.N, dim=d.dim, ic=kind, seed=seed, No_Ek_plot=n_ek, steps=rec["steps"], t_final=t,
                dt_final=float(d.dt))
    out["meta"] = np.array(json.dumps(meta))
    return out


def run_diag(ref):
    """U_square and dissipation_rate (src/RK4_method.py:77-101) and the
    calculate_Ek bins (src/SM_solver.py:94-192) on seeded 3D and 2D fields."""
    sm = ref["SM_solver"]
    rk4 = ref["RK4_method"]
    D = ref["initialize_domain"].InitializeDomain
    out = {}
    for tag, kw, ic in (("rand16", dict(No_of_gridpoint=16, dimension=3, nu=1e-2, method="RK4"), ("rand", 41)),
                        ("noise16", dict(No_of_gridpoint=16, dimension=3, nu=3e-3, method="RK4"), ("noise", 42)),
                        ("vort32", dict(No_of_gridpoint=32, dimension=2, nu=1e-3, method="RK4"), ("vort", 43))):
        d = D(**kw)
        kind, seed = ic
        if kind == "vort":
            (omega,) = _ic(kind, d.N, d.dim, seed, mean=0.0)
            ref["initial"].initial_vorticity(d, omega)
            out[tag + "_omega0"] = omega
        else:
            f = _ic(kind, d.N, d.dim, seed)
            ref["initial"].initial_velocity(d, *f)
            out[tag + "_u0"] = np.array(f)
        out[tag + "_U_square"] = np.array(rk4.U_square(d))
        out[tag + "_dissipation_rate"] = np.array(rk4.dissipation_rate(d))
        E = sm.Ek_plot_variables.__new__(sm.Ek_plot_variables)
        # Ek_plot_variables.__init__ minus its plot and CSV set-up (src/SM_solver.py:94-112)
        E.Ek = np.empty(np.array(d.P_hat).shape, dtype=float)
        d.k2 = np.unique(d.K2)
        if d.dim == 2:
            K2 = np.array(np.meshgrid(d.kx, d.kz, indexing="ij"), dtype=int)
        else:
            K2 = np.array(np.meshgrid(d.kx, d.kx.copy(), d.kz, indexing="ij"), dtype=int)
        K2 = np.sum(K2 * K2, 0, dtype=int)
        E.avgPara = 5
        E.smoothing_para = round(np.sqrt(np.max(np.unique(K2)))) // E.avgPara
        E.temp_k = np.zeros(E.smoothing_para + 1)
        E.temp_Ek = np.zeros(E.smoothing_para + 1)
        sm.calculate_Ek(d, E)
        out[tag + "_temp_k"] = E.temp_k.copy()
        out[tag + "_temp_Ek"] = E.temp_Ek.copy()
        out[tag + "_meta"] = np.array(json.dumps(dict(kw, N=d.N, ic=kind, seed=seed)))
    return out


def main(argv=None):
    import argparse
    global REF
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=REF, help="path of a reference checkout (holds src/)")
    ap.add_argument("--only", default="steps,ops,solver,diag", help="fixture groups to write")
    a = ap.parse_args(argv)
    REF = a.reference
    groups = set(a.only.split(","))
    ref = import_reference()
    if "ops" in groups:
        np.savez_compressed(os.path.join(HERE, "ops16.npz"), **run_ops(ref))
    if "diag" in groups:
        np.savez_compressed(os.path.join(HERE, "diag16.npz"), **run_diag(ref))
        print("wrote diag16")
    if "steps" in groups:
        for name, kw, ic, steps in CASES:
            out = run_case(ref, name, kw, ic, steps)
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
            print("wrote", name, {k: v.shape for k, v in out.items() if k != "meta"})
    if "solver" in groups:
        for name, kw, ic, n_ek in SOLVER_CASES:
            out = run_solver(ref, name, kw, ic, n_ek)
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
            print("wrote", name, json.loads(str(out["meta"]))["steps"], "steps")


if __name__ == "__main__":
    main()
