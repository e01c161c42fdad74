#!/usr/bin/env python
"""Throughput benchmark: grid-point*steps/s of the fused FP32 path.

Workload (the reference-scale LES case): decaying isotropic turbulence LES on a
2pi-periodic 256^3 grid, seeded random-phase spectrum (k0=4, u0=1, seed 0),
nu=1e-4, Smagorinsky Cs=0.17 with Delta=2pi/256, the reference's RK3 scheme,
dt=1e-3.  One "step" = one RK3 step (3 fused RHS evaluations + stage updates).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sles|reference]

Under torchrun each rank advances its own ensemble member (seed = rank) with no
data-path collective; value = points*steps of all ranks / max-over-ranks time.
Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "spectral-les_b200"))
sys.path.insert(0, REPO)

METRIC = "Mpts·steps/s at 256³/512³, FP32 fused vs FP64 GPU at stated err; adjoint/fwd ratio"
UNIT = "Mpts·steps/s"
NU, CS, DT, K0, U0 = 1e-4, 0.17, 1e-3, 4.0, 1.0
# algorithmic HBM bytes per grid point per RHS evaluation (3D LES, FP32): 21 transforms
# x 16 B (two out-of-cache passes, read+write) + 48 B integrator state
STEP_BYTES_PER_PT_RHS = {"f32": 384.0, "f64": 768.0}
TUNE = True  # run the autotuner on each timed domain (outside the timed regions)


def workload_name(n):
    return ("decaying isotropic turbulence LES %d^3, Smagorinsky Cs=%.2f (Delta=2pi/%d), reference RK3, "
            "dt=%g, nu=%g, random-phase spectrum k0=%g u0=%g" % (n, CS, n, DT, NU, K0, U0))


def bench_config(n, world):
    """The workload description both arms print (identical dicts)."""
    fbytes = float(n) * n * (n // 2 + 1) * 8
    return {"workload": workload_name(n), "n": n, "scheme": "RK3 (reference arithmetic)", "les": "Smagorinsky",
            "l2": "inputs larger than L2 (state 3x3x%.0f MB + workspace 9 fields at FP32)" % (fbytes / 1e6),
            "parallelism": "replicas" if world > 1 else "single device"}


def measured_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    return 6650.0, "fallback 6.65 TB/s"


def ncu_traffic(kernel_key):
    p = os.path.join(REPO, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f).get(kernel_key)


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", "sles_clocks_%d.csv" % os.getpid())

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[2], parts[3:]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["active_mask", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for nm, v in zip(names[1:], r[3][1:]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "samples": len(rows), "reasons": sorted(reasons)}


def gpu_index():
    import torch
    try:
        props = torch.cuda.get_device_properties(torch.cuda.current_device())
        bus = "%08x:%02x:%02x.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
        out = subprocess.run(["nvidia-smi", "--query-gpu=index,pci.bus_id", "--format=csv,noheader"],
                             capture_output=True, text=True, timeout=20).stdout
        for line in out.splitlines():
            idx, b = [x.strip() for x in line.split(",")]
            if b.lower().endswith(bus[-7:].lower()):
                return int(idx)
    except Exception:
        pass
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]
    return int(vis) if vis.isdigit() else 0


# ---------------------------------------------------------------------------
# the fused path
# ---------------------------------------------------------------------------
def make_domain(n, dtype, seed, method="RK3", les="Smagorinsky", nu=NU, cs=CS, dt=DT, k0=K0, parity=True):
    import torch
    from sles.initialize_domain import InitializeDomain
    from sles.initial import initial_velocity
    from sles.synthetic import random_spectrum_velocity
    d = InitializeDomain(nu=nu, dimension=3, time_stepSize=dt, No_of_gridpoint=(4 if les else 1) * n, method=method,
                         LES_ON=1 if les else 0, LES_model=les, Cs=cs, dtype=dtype, parity_mode=parity)
    u, v, w = random_spectrum_velocity(n, k0, U0, seed=seed)
    initial_velocity(d, u, v, w)
    del u, v, w
    torch.cuda.synchronize()
    return d


def spectrum_error(a, b, n, floor=1e-8):
    """E(k) error of a against b on integer shells 1..floor(2/3 (N/2+1)):
    (max relative error over the shells holding at least ``floor`` of the peak
    shell energy, the last such shell, max relative error over all shells).
    Shells far below the peak carry round-off-level energy in float32, where
    the relative error measures the float32 noise floor, not the dynamics."""
    from sles.adjoint import shell_spectrum
    kc = int(2.0 / 3.0 * (n // 2 + 1))
    ea, eb = shell_spectrum(a, n, kc + 1)[1:], shell_spectrum(b, n, kc + 1)[1:]
    r = (ea - eb).abs() / eb
    live = eb >= floor * eb.max()
    klast = int(live.nonzero().max()) + 1
    return float(r[live].max()), klast, float(r.max())


def error_history(d32, d64, step, nsteps, n, every=None):
    """Step both domains ``nsteps`` times, recording after every step the
    relative L2 velocity error of the float32 state against the float64 one
    and the E(k) error (shells above 1e-8 of the peak).  Returns the maxima,
    the final values and a thinned series."""
    every = every or max(1, nsteps // 10)
    l2, ek = [], []
    for _ in range(nsteps):
        step(d32)
        step(d64)
        l2.append(rel_l2(d32.U_hat, d64.U_hat))
        ek.append(spectrum_error(d32.U_hat, d64.U_hat, n)[0])
    return {"steps": nsteps, "rel_l2_max": max(l2), "rel_l2_final": l2[-1], "ek_err_max": max(ek),
            "ek_err_final": ek[-1], "rel_l2_every_%d" % every: [float("%.3g" % x) for x in l2[every - 1::every]],
            "ek_err_every_%d" % every: [float("%.3g" % x) for x in ek[every - 1::every]]}


def bench_cfg2_history(rank, steps=500):
    """The Smagorinsky LES workload at 256^3 (reference RK3, dt = 1e-3) run
    for its 500 steps in float32 and in float64 (the oracle precision), with
    the velocity and E(k) errors recorded after every step."""
    import torch
    from sles import RK3_method
    d32 = make_domain(256, "float32", rank)
    d64 = make_domain(256, "float64", rank)
    out = error_history(d32, d64, RK3_method.solveForNextTimestep, steps, 256, every=50)
    d32._plan.check()
    d64._plan.check()
    del d32, d64
    torch.cuda.empty_cache()
    out["config"] = "256^3 Smagorinsky Cs=0.17, nu=1e-4, reference RK3, dt=1e-3, seed = rank; float32 vs float64 fused"
    return out


def bench_cfg1(rank):
    """The plain Taylor-Green case: 64^3, nu = 1/1600, RK4, dt = 0.01, 200
    steps, float64, no LES; kinetic energy and dissipation every step (the
    reference's U_square / dissipation_rate outputs, here as E = 1/2 <u.u>
    and eps = nu <|grad u|^2>).  Reports the rate, E(t) against the analytic
    early decay 1/8 exp(-6 nu t) over t <= 0.2, and the energy budget
    dE/dt + eps relative to eps."""
    import numpy as np
    import torch
    from sles import RK4_method, diagnostics
    from sles.initial import initial_velocity
    from sles.initialize_domain import InitializeDomain
    from sles.synthetic import taylor_green
    n, nu, dt, steps = 64, 1.0 / 1600.0, 0.01, 200
    d = InitializeDomain(nu=nu, dimension=3, time_stepSize=dt, No_of_gridpoint=n, method="RK4", dtype="float64")
    initial_velocity(d, *taylor_green(n))
    d.U_hat1[...] = d.U_hat
    E, eps = [diagnostics.energy(d)], [diagnostics.dissipation(d)]
    secs = 0.0
    for _ in range(steps):
        secs += time_steps(d, 1, RK4_method.solveForNextTimestep)
        E.append(diagnostics.energy(d))
        eps.append(diagnostics.dissipation(d))
    d._plan.check()
    E, eps = np.array(E), np.array(eps)
    t = np.arange(steps + 1) * dt
    early = t <= 0.2 + 1e-12
    exact = 0.125 * np.exp(-6 * nu * t)
    budget = np.abs((E[2:] - E[:-2]) / (2 * dt) + eps[1:-1]) / eps[1:-1]
    return {"value": round(float(n) ** 3 * steps / secs / 1e6, 2), "unit": UNIT, "steps": steps,
            "E_0": E[0], "E_end": E[-1], "eps_0": eps[0], "eps_end": eps[-1],
            "E_rel_dev_from_exp_decay_t_le_0.2": float(np.max(np.abs(E[early] - exact[early]) / exact[early])),
            "energy_budget_rel_err_max": float(budget.max()),
            "config": "Taylor-Green 64^3, nu=1/1600, RK4, dt=0.01, 200 steps, float64, no LES; E and eps every step"}


def tune_domain(d):
    """Run the autotuner on a domain (outside any timed region); the cache goes
    to a per-process temporary file unless SLES_TUNE_CACHE is set."""
    import tempfile
    from sles import autotune
    if not os.environ.get("SLES_TUNE_CACHE"):
        os.environ["SLES_TUNE_CACHE"] = os.path.join(tempfile.gettempdir(), "sles_bench_tune_%d.json" % os.getpid())
    report = autotune.tune(d) if TUNE else {}
    names = {0: "x", 1: "y", 2: "z"}
    return {"variants": {names[p]: d._plan.get_variant(p) for p in names},
            "ms_per_step_by_variant": {names[p]: {str(k): round(v, 4) for k, v in t.items()}
                                       for p, t in report.items()}}


def rel_l2(a, b):
    import torch
    return float(torch.linalg.vector_norm(a.to(b.dtype) - b) / torch.linalg.vector_norm(b))


def bench_512(peak, rank):
    """512^3 cases: the Smagorinsky LES recipe (RK3, cfg-2 parameters) at 512^3
    against the plain FP64 GPU path and FP64 fused after 100 steps; and the
    Vreman ETD2 case (k0=6, nu=5e-5, c=0.07 i.e. Cs=sqrt(0.028), dt=5e-4,
    corrected ETD2 with float64 phi-coefficients), FP32 against FP64 after 100
    steps, with per-kernel times."""
    import torch
    from sles import ETD2_method, RK3_method
    n, npts, out = 512, 512.0 ** 3, {}
    step = RK3_method.solveForNextTimestep
    # -- Smagorinsky RK3 at 512^3
    d32 = make_domain(n, "float32", rank)
    d64 = make_domain(n, "float64", rank)
    tu = [tune_domain(d32), tune_domain(d64)]
    for _ in range(3):
        step(d32)
        step(d64)
    t32 = time_steps(d32, 20, step)
    t64 = time_steps(d64, 20, step)
    hist = error_history(d32, d64, step, 100 - 23, n)
    err = rel_l2(d32.U_hat, d64.U_hat)
    ek, klive, ekall = spectrum_error(d32.U_hat, d64.U_hat, n)
    kms = d32._plan.profile_rhs(d32._s_uhat, d32._new_hc(3), 10)
    del d32, d64
    torch.cuda.empty_cache()
    tp = torch_plain_fp64_rk3(n, 2, 1, rank)
    torch.cuda.empty_cache()
    v32, v64, vtp = npts * 20 / t32 / 1e6, npts * 20 / t64 / 1e6, npts / tp / 1e6
    ms = t32 / 20 * 1e3
    names = ["x_inverse", "y_inverse", "z_fused", "y_forward", "x_forward_combine"]
    fbytes = float(n) * n * (n // 2 + 1) * 8
    algb = {"x_inverse": 9 * fbytes, "y_inverse": 15 * fbytes, "z_fused": 18 * fbytes, "y_forward": 15 * fbytes,
            "x_forward_combine": 18 * fbytes}
    out["smagorinsky_rk3"] = {
        "value": round(v32, 2), "unit": UNIT, "ms_per_step": round(ms, 3),
        "fused_fp64_value": round(v64, 2), "torch_fft_fp64_value": round(vtp, 2),
        "speedup_vs_torch_fp64": round(v32 / vtp, 2), "speedup_vs_fused_fp64": round(v32 / v64, 2),
        "rel_l2_fp32_vs_fp64_after_100_steps": err,
        "ek_err_fp32_vs_fp64_after_100_steps": {"max_rel_shells_above_1e-8_of_peak": ek, "up_to_shell": klive,
                                                "max_rel_all_shells": ekall},
        "error_every_step_24_to_100": hist,
        "step_roofline_frac": round(STEP_BYTES_PER_PT_RHS["f32"] * 3 * npts / (ms * 1e-3) / 1e9 / peak, 4),
        "kernel_ms": dict(zip(names, [round(x, 4) for x in kms])),
        "kernel_gbs": {k: round(algb[k] / (t * 1e-3) / 1e9, 1) for k, t in zip(names, kms)},
        "autotune_fp32_fp64": tu,
        "config": "512^3, random-phase spectrum k0=4, nu=1e-4, Smagorinsky Cs=0.17, reference RK3, dt=1e-3"}
    # -- Vreman ETD2 at 512^3
    cs_v = math.sqrt(0.07 / 2.5)
    mk = lambda dt_: make_domain(n, dt_, rank, method="ETD2", les="vreman", nu=5e-5, cs=cs_v, dt=5e-4, k0=6.0,
                                 parity=False)
    estep = ETD2_method.solveForNextTimestep
    d32, d64 = mk("float32"), mk("float64")
    tu = [tune_domain(d32), tune_domain(d64)]
    for _ in range(3):
        estep(d32)
        estep(d64)
    t32 = time_steps(d32, 20, estep)
    t64 = time_steps(d64, 20, estep)
    hist = error_history(d32, d64, estep, 100 - 23, n)
    err = rel_l2(d32.U_hat, d64.U_hat)
    ek, klive, ekall = spectrum_error(d32.U_hat, d64.U_hat, n)
    kms = d32._plan.profile_rhs(d32._s_uhat, d32._new_hc(3), 10)
    fbytes = float(n) * n * (n // 2 + 1) * 8
    algb = {"x_inverse": 9 * fbytes, "y_inverse": 15 * fbytes, "z_fused": 18 * fbytes, "y_forward": 15 * fbytes,
            "x_forward_combine": 18 * fbytes}
    names = ["x_inverse", "y_inverse", "z_fused", "y_forward", "x_forward_combine"]
    del d32, d64
    torch.cuda.empty_cache()
    ms = t32 / 20 * 1e3
    out["vreman_etd2"] = {
        "value": round(npts * 20 / t32 / 1e6, 2), "unit": UNIT, "ms_per_step": round(ms, 3),
        "fused_fp64_value": round(npts * 20 / t64 / 1e6, 2),
        "rel_l2_fp32_vs_fp64_after_100_steps": err,
        "ek_err_fp32_vs_fp64_after_100_steps": {"max_rel_shells_above_1e-8_of_peak": ek, "up_to_shell": klive,
                                                "max_rel_all_shells": ekall},
        "error_every_step_24_to_100": hist,
        "step_roofline_frac": round(STEP_BYTES_PER_PT_RHS["f32"] * 1 * npts / (ms * 1e-3) / 1e9 / peak, 4),
        "kernel_ms": dict(zip(names, [round(x, 4) for x in kms])),
        "kernel_gbs": {k: round(algb[k] / (t * 1e-3) / 1e9, 1) for k, t in zip(names, kms)},
        "autotune_fp32_fp64": tu,
        "config": "512^3, random-phase spectrum k0=6, nu=5e-5, Vreman c=0.07 (Cs=%.5f), ETD2 (Cox-Matthews, "
                  "float64 phi coefficients), dt=5e-4" % cs_v}
    return out


def time_steps(d, k, step):
    import torch
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(k):
        step(d)
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3


def torch_plain_fp64_rk3(n, steps, warmup, seed):
    """The plain FP64 GPU path: the reference's RK3 + Smagorinsky RHS written
    with torch.fft (cuFFT) and unfused elementwise ops (no custom kernels)."""
    import torch
    from sles.synthetic import random_spectrum_velocity
    dev = "cuda"
    kc = torch.fft.fftfreq(n, 1.0 / n, device=dev, dtype=torch.float64).round()
    kr = kc[: n // 2 + 1].clone()
    kr[-1] = -kr[-1]
    K = [kc.view(n, 1, 1), kc.view(1, n, 1), kr.view(1, 1, -1)]
    K2 = K[0] ** 2 + K[1] ** 2 + K[2] ** 2
    KoK2 = [k / torch.where(K2 == 0, torch.ones_like(K2), K2) for k in K]
    kmax = 2.0 / 3.0 * (n // 2 + 1)
    mask = ((K[0].abs() < kmax) & (K[1].abs() < kmax) & (K[2].abs() < kmax)).to(torch.float64)
    dx = 2 * math.pi / n
    f = lambda a: torch.fft.rfftn(a, dim=(-3, -2, -1))
    b = lambda a: torch.fft.irfftn(a, s=(n, n, n), dim=(-3, -2, -1))

    def rhs(Uh):
        U = b(Uh)
        curl = torch.stack([b(1j * (K[1] * Uh[2] - K[2] * Uh[1])), b(1j * (K[2] * Uh[0] - K[0] * Uh[2])),
                            b(1j * (K[0] * Uh[1] - K[1] * Uh[0]))])
        dU = torch.stack([f(U[1] * curl[2] - U[2] * curl[1]), f(U[2] * curl[0] - U[0] * curl[2]),
                          f(U[0] * curl[1] - U[1] * curl[0])]) * mask
        A = [[b(1j * K[i] * Uh[j]) for j in range(3)] for i in range(3)]
        ss = sum(A[i][i] ** 2 for i in range(3)) + sum(0.5 * (A[i][j] + A[j][i]) ** 2 for i in range(3)
                                                       for j in range(i + 1, 3))
        nu_t = torch.sqrt(2.0 * ss) * (CS * dx) ** 2
        S = lambda i, j: A[i][i] if i == j else 0.5 * (A[i][j] + A[j][i])
        T = torch.stack([sum(K[j] * f(S(i, j) * nu_t) for j in range(3)) * (2j * mask) for i in range(3)])
        P = sum((dU[i] + T[i]) * KoK2[i] for i in range(3))
        dU = torch.stack([dU[i] - P * K[i] for i in range(3)])
        return dU - NU * K2 * Uh + T

    u, v, w = random_spectrum_velocity(n, K0, U0, seed=seed)
    Uh = f(torch.stack([u, v, w]))

    def step(Uh):
        U0_ = Uh
        dU = rhs(Uh)
        Uh = U0_ + 0.5 * DT * dU
        dU = rhs(Uh)
        Uh = U0_ - DT * dU + 2.0 * DT * dU
        dU = rhs(Uh)
        return U0_ + DT * (1 / 6 * dU + 2 / 3 * dU + 1 / 6 * dU)

    for _ in range(warmup):
        Uh = step(Uh)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        Uh = step(Uh)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / steps


def cpu_oracle_rate(n, steps, warmup, seed, workers):
    """The oracle (NumPy/SciPy restatement of the reference) on the host cores."""
    from oracle import spectral_oracle as so
    so.set_fft_workers(workers)
    o = so.OracleDomain(n, 3, nu=NU, dt=DT, les_model="Smagorinsky", Cs=CS, method="RK3")
    so.initial_velocity(o, *so.random_spectrum_velocity(n, K0, U0, seed=seed))
    for _ in range(warmup):
        so.step(o)
    t0 = time.perf_counter()
    for _ in range(steps):
        so.step(o)
    dt = time.perf_counter() - t0
    so.set_fft_workers(None)
    return n ** 3 * steps / dt / 1e6, dt


def max_over_ranks_of(x, world, device):
    """The maximum of a per-rank float over all ranks of the default process group."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(points_per_rank, steps, secs_local, world, device):
    """Whole-job Mpts*steps/s of ``world`` replicas (each rank advances its own
    member of ``points_per_rank`` points): all ranks' points over the slowest
    rank's time.  Returns (value, max seconds)."""
    secs = max_over_ranks_of(secs_local, world, device)
    return world * points_per_rank * steps / secs / 1e6, secs


def run_reference(args, rank, world):
    """The reference arm: the oracle port of the reference's RK3 + Smagorinsky
    path (float64 NumPy, scipy.fft with a worker per host core) on a bounded
    sample of the same workload; its rate stands for the requested steps."""
    if rank != 0:
        return
    n = args.n
    cores = os.cpu_count() or 1
    w = min(args.warmup, 1)
    k = max(1, min(args.steps, 2))
    value, secs = cpu_oracle_rate(n, k, w, 0, cores)
    sample = ("%d timed RK3 step(s) at %d^3 after %d warm-up step(s); the rate stands for the requested %d "
              "steps (%.0f s at %.1f s/step, extrapolated); oracle port (NumPy + scipy.fft workers=%d) on the "
              "host cores; the reference itself needs mpi4py/mpi4py-fft, absent on this image (its own src/ "
              "under a single-rank shim with the same threaded FFTs took 0.88x the port's time per step at "
              "256^3 on an 8-core CPU: oracle/time_reference.py)" % (k, n, w, args.steps, secs / k * args.steps,
                                                                     secs / k, cores))
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
           "steps": k, "steps_requested": args.steps, "warmup": w, "ms_per_step": round(secs / k * 1e3, 2),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded random-phase spectrum, seed=rank)", "config": bench_config(n, world),
           "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": cores, "kind": "port",
                            "sample": sample},
           "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def bench_fft(rank):
    """The project's batched 3D r2c / c2r (sles_fft_r2c / sles_fft_c2r, 3
    fields) against torch.fft.rfftn / irfftn (cuFFT) on the same 3 fields, at
    256^3 and 512^3 in float32 and float64: mean ms per call (CUDA events, 10
    calls after 3 warm-up calls) and the effective HBM rate of a two-pass
    out-of-cache transform model (real read + half-complex written, twice)."""
    import torch
    from sles import _native as nat
    out = {}
    for n in (256, 512):
        for dt in (torch.float32, torch.float64):
            tag = "%d_%s" % (n, "f32" if dt == torch.float32 else "f64")
            plan = nat.Plan(3, n, dt, nat.LES_NONE, nat.SCHEME_RK4, True, 0.0, 0.0, 0.0, "cuda")
            g = torch.Generator(device="cuda").manual_seed(rank)
            x = torch.randn((3, n, n, n), dtype=dt, device="cuda", generator=g)
            cd = torch.complex64 if dt == torch.float32 else torch.complex128
            hc = torch.empty((3, n, n, plan.nkp), dtype=cd, device="cuda")
            y = torch.empty_like(x)

            def timeit(fn, reps=10):
                for _ in range(3):
                    fn()
                st = torch.cuda.current_stream()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(st)
                for _ in range(reps):
                    fn()
                e1.record(st)
                torch.cuda.synchronize()
                return e0.elapsed_time(e1) / reps

            r = {"sles_r2c_ms": timeit(lambda: plan.fft_r2c(x, hc, 3)),
                 "sles_c2r_ms": timeit(lambda: plan.fft_c2r(hc, y, 3))}
            err_rt = float(torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x))
            ref = torch.fft.rfftn(x, dim=(1, 2, 3))
            err_f = float(torch.linalg.vector_norm(hc[..., : n // 2 + 1] - ref) / torch.linalg.vector_norm(ref))
            del ref
            r["cufft_rfftn_ms"] = timeit(lambda: torch.fft.rfftn(x, dim=(1, 2, 3)))
            h2 = torch.fft.rfftn(x, dim=(1, 2, 3))
            r["cufft_irfftn_ms"] = timeit(lambda: torch.fft.irfftn(h2, s=(n, n, n), dim=(1, 2, 3)))
            del h2
            esz = 4 if dt == torch.float32 else 8
            model = 3 * 2 * (float(n) ** 3 * esz + float(n) * n * (n // 2 + 1) * 2 * esz)
            for k in ("sles_r2c_ms", "sles_c2r_ms", "cufft_rfftn_ms", "cufft_irfftn_ms"):
                r[k] = round(r[k], 4)
            r["sles_r2c_gbs"] = round(model / (r["sles_r2c_ms"] * 1e-3) / 1e9, 1)
            r["cufft_rfftn_gbs"] = round(model / (r["cufft_rfftn_ms"] * 1e-3) / 1e9, 1)
            r["speedup_r2c_vs_cufft"] = round(r["cufft_rfftn_ms"] / r["sles_r2c_ms"], 3)
            r["speedup_c2r_vs_cufft"] = round(r["cufft_irfftn_ms"] / r["sles_c2r_ms"], 3)
            r["rel_err_r2c_vs_cufft"] = err_f
            r["rel_err_roundtrip"] = err_rt
            out[tag] = r
            del x, y, hc, plan
            torch.cuda.empty_cache()
    out["note"] = ("3 fields per call; the project's transforms are the unfused standalone passes (r2c lines, "
                   "then c2c along y and x); the fused RHS never runs them")
    return out


def bench_adjoint(rank):
    """Adjoint case: 128^3 Smagorinsky LES, RK4, nu=2e-4, dt=2e-3, 100 steps,
    FP32 forward and FP32 adjoint with checkpoints every 10 steps.  Loss
    sum_k (log E(k,T) - log E_target(k))^2 over shells 1..43; E_target from a
    256^3 FP64 no-LES RK4 run of the same recipe and seed to T=0.2 (shells
    1..43 lie inside the 128^3 dealiased band).  Reports forward and backward
    times (CUDA events) and the gradients' agreement with the FP64 adjoint and
    with a central difference in Cs (eps=1e-3, FP64)."""
    import torch
    from sles import RK4_method
    from sles.adjoint import ETD2Rollout, RK3Rollout, RK4Rollout, log_spectrum_misfit, shell_spectrum
    n, nu, dt, steps, cs = 128, 2e-4, 2e-3, 100, CS
    dT = make_domain(256, "float64", rank, method="RK4", les=None, nu=nu, dt=dt)
    dT.U_hat1[...] = dT.U_hat
    for _ in range(steps):
        RK4_method.solveForNextTimestep(dT)
    Et = shell_spectrum(dT.U_hat, 256, 44).detach()
    del dT
    d0 = make_domain(n, "float64", rank, method="RK4", nu=nu, dt=dt)
    U0 = d0.U_hat.clone()
    tune_domain(d0)
    del d0
    d1 = make_domain(n, "float32", rank, method="RK4", nu=nu, dt=dt)
    tune_domain(d1)
    del d1
    res = {}
    for name, dtp in (("f32", torch.float32), ("f64", torch.float64)):
        ro = RK4Rollout(n, nu, dt, les="Smagorinsky", Cs=cs, dtype=dtp, checkpoint_every=10)
        U = U0.to(ro.cdtype)
        # gradient of the loss at U_T (torch autograd on the loss only), then timed sweeps
        UT, _ = ro.forward_states(U, cs, steps)
        UTv = UT[..., : ro.nk].clone().requires_grad_(True)
        loss = log_spectrum_misfit(UTv, Et, n)
        gUT, = torch.autograd.grad(loss, [UTv])
        ro.timed(U, cs, steps, gUT)  # warm-up (allocations)
        fw, bw = [], []
        for _ in range(3):
            f_ms, b_ms, _, g, c = ro.timed(U, cs, steps, gUT)
            fw.append(f_ms)
            bw.append(b_ms)
        res[name] = dict(fwd_ms=min(fw), bwd_ms=min(bw), loss=float(loss.detach()), g=g[..., : ro.nk].to(torch.complex128),
                         cs=float(c[0]), ro=ro, U=U)
    r32, r64 = res["f32"], res["f64"]
    # the reference's RK3 with its adjoint, same recipe in FP32
    ro3 = RK3Rollout(n, nu, dt, les="Smagorinsky", Cs=cs, dtype=torch.float32, checkpoint_every=10)
    U3 = U0.to(ro3.cdtype)
    UT3 = ro3.forward_states(U3, cs, steps)[0][..., : ro3.nk].clone().requires_grad_(True)
    gUT3, = torch.autograd.grad(log_spectrum_misfit(UT3, Et, n), [UT3])
    ro3.timed(U3, cs, steps, gUT3)
    t3 = [ro3.timed(U3, cs, steps, gUT3)[:2] for _ in range(3)]
    f3, b3 = min(t[0] for t in t3), min(t[1] for t in t3)
    del ro3, U3, UT3, gUT3
    # the corrected ETD2 with its adjoint, same recipe in FP32
    roe = ETD2Rollout(n, nu, dt, les="Smagorinsky", Cs=cs, dtype=torch.float32, checkpoint_every=10)
    Ue = U0.to(roe.cdtype)
    UTe = roe.forward_states(Ue, cs, steps)[0][..., : roe.nk].clone().requires_grad_(True)
    gUTe, = torch.autograd.grad(log_spectrum_misfit(UTe, Et, n), [UTe])
    st = torch.cuda.current_stream()
    te = []
    for _ in range(4):  # the first is a warm-up
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        ev[0].record(st)
        _, ck = roe.forward_states(Ue, cs, steps)
        ev[1].record(st)
        roe.backward_states(ck, gUTe, cs, steps)
        ev[2].record(st)
        torch.cuda.synchronize()
        te.append((ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])))
        del ck
    fe, be = min(t[0] for t in te[1:]), min(t[1] for t in te[1:])
    del roe, Ue, UTe, gUTe
    # central difference in Cs on the FP64 path
    ro, U = r64["ro"], r64["U"]
    lo = lambda c: float(log_spectrum_misfit(ro.forward_states(U, c, steps)[0][..., : ro.nk], Et, n))
    cd = lambda e: (lo(cs + e) - lo(cs - e)) / (2 * e)
    fd1, fd2 = cd(1e-3), cd(5e-4)
    fd = (4.0 * fd2 - fd1) / 3.0  # Richardson: O(eps^4) truncation
    g32, g64 = r32["g"], r64["g"]
    out = {"fwd_ms": round(r32["fwd_ms"], 2), "bwd_ms": round(r32["bwd_ms"], 2),
           "adjoint_fwd_ratio": round(r32["bwd_ms"] / r32["fwd_ms"], 3),
           "fwd_ms_f64": round(r64["fwd_ms"], 2), "bwd_ms_f64": round(r64["bwd_ms"], 2),
           "adjoint_fwd_ratio_f64": round(r64["bwd_ms"] / r64["fwd_ms"], 3),
           "loss": r32["loss"], "dL_dCs_f32": r32["cs"], "dL_dCs_f64": r64["cs"], "dL_dCs_central_diff_f64_eps1e-3": fd1,
           "dL_dCs_richardson_f64": fd, "cs_rel_err_f64_vs_richardson": abs(r64["cs"] - fd) / abs(fd),
           "cs_rel_err_f32_vs_richardson": abs(r32["cs"] - fd) / abs(fd),
           "grad_u0_rel_l2_f32_vs_f64": rel_l2(g32, g64),
           "rk3": {"fwd_ms": round(f3, 2), "bwd_ms": round(b3, 2), "adjoint_fwd_ratio": round(b3 / f3, 3),
                   "scheme": "the reference's RK3 (3 stages), FP32, same recipe"},
           "etd2": {"fwd_ms": round(fe, 2), "bwd_ms": round(be, 2), "adjoint_fwd_ratio": round(be / fe, 3),
                    "scheme": "corrected ETD2 (first step RK4), FP32, same recipe, checkpoints every 10"},
           "config": "128^3, random-phase spectrum k0=4, nu=2e-4, Smagorinsky Cs=0.17, RK4, dt=2e-3, 100 steps, "
                     "checkpoints every 10, loss on log E(k), k=1..43; backward = segment recompute + reverse stages"}
    del res, r32, r64, ro, U
    torch.cuda.empty_cache()
    return out


def bench_driver(rank, n=128, t_end=4.0):
    """The driver loop (SM_solver.spectralMethodSolver, adaptive CFL dt, E(k)
    snapshots) with its time-step logic on the host (a device->host read of
    max u every step) against device_dt=True (dt on the GPU, steps replayed as
    graph chunks): 128^3 FP32 Smagorinsky, reference RK3, CFL 0.5, wall time."""
    import tempfile
    import torch
    from sles.SM_solver import spectralMethodSolver
    out = {}
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as td:
        os.chdir(td)
        try:
            for mode in (False, True, False, True):  # the first pair warms up
                d = make_domain(n, "float32", rank)
                d.T, d.CFL = t_end, 0.5
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                steps = spectralMethodSolver(d, No_Ek_plot=5, verbose=False, device_dt=mode, chunk=32)
                torch.cuda.synchronize()
                secs = time.perf_counter() - t0
                out["device_dt" if mode else "host_dt"] = {
                    "steps": steps, "wall_s": round(secs, 4), "final_dt": d.dt,
                    "value": round(float(n) ** 3 * steps / secs / 1e6, 2), "unit": UNIT}
                del d
        finally:
            os.chdir(cwd)
    out["speedup_device_dt"] = round(out["device_dt"]["value"] / out["host_dt"]["value"], 3)
    out["config"] = ("%d^3 FP32 Smagorinsky Cs=0.17, reference RK3, nu=1e-4, CFL 0.5 (0.3 first step), final "
                     "time %g, 5 E(k) snapshots; wall time of spectralMethodSolver including its set-up" % (n, t_end))
    return out


def ensemble_members(seed):
    """48 members from one generator: 32 2D vorticity runs (N in {256, 512,
    1024}, nu log-uniform in [1e-5, 1e-3], Gaussian vorticity peaked at k=10,
    RK4, dt=1e-3) and 16 3D Smagorinsky runs (N in {64, 96, 128}, Cs uniform
    in [0.1, 0.2], random-phase spectrum k0=4, nu=1e-4, RK4, dt=1e-3); FP32."""
    import numpy as np
    from sles.initial import initial_velocity, initial_vorticity
    from sles.initialize_domain import InitializeDomain
    from sles.synthetic import gaussian_vorticity_2d, random_spectrum_velocity
    rng = np.random.default_rng(seed)
    members = []
    for i in range(32):
        n = int(rng.choice([256, 512, 1024]))
        nu = float(10.0 ** rng.uniform(-5, -3))
        d = InitializeDomain(nu=nu, dimension=2, time_stepSize=1e-3, No_of_gridpoint=n, method="RK4",
                             dtype="float32")
        initial_vorticity(d, gaussian_vorticity_2d(n, seed=int(rng.integers(1 << 30)), kp=10.0))
        members.append(d)
    for i in range(16):
        n = int(rng.choice([64, 96, 128]))
        cs = float(rng.uniform(0.1, 0.2))
        d = InitializeDomain(nu=NU, dimension=3, time_stepSize=1e-3, No_of_gridpoint=4 * n, method="RK4", LES_ON=1,
                             LES_model="Smagorinsky", Cs=cs, dtype="float32")
        initial_velocity(d, *random_spectrum_velocity(n, K0, U0, seed=int(rng.integers(1 << 30))))
        members.append(d)
    for d in members:
        d.U_hat1[...] = d.U_hat
    return members


def bench_slab(rank, n=512, nranks=(2, 4), steps=3):
    """The slab decomposition's compute on one GPU: the P ranks of one 512^3
    FP32 Smagorinsky RK3 domain run one after another in one process (their
    all-to-alls as copies between their buffers, outside the timed calls).
    Each rank's own kernel time per step (CUDA events around its prime,
    middle and stage calls) against the whole-grid fused step, and the bytes
    each rank sends per step through the two exchanges of every RHS
    evaluation.  The projected multi-GPU step (the slowest rank's compute plus
    its exchange bytes at the measured 770 GB/s per direction of a peer copy,
    not overlapped) is a model, not a measurement."""
    import torch
    from sles import RK3_method
    from sles.slab import SlabDomain
    d = make_domain(n, "float32", rank)
    U = d.U_hat.clone()
    whole = time_steps(d, steps, RK3_method.solveForNextTimestep)
    del d
    torch.cuda.empty_cache()
    out = {"n": n, "whole_grid_ms_per_step": round(whole / steps * 1e3, 3)}
    st = torch.cuda.current_stream()
    for P in nranks:
        doms = [SlabDomain(n, nu=NU, dt=DT, method="RK3", les="Smagorinsky", Cs=CS, dtype=torch.float32, nranks=P,
                           rank=r, exchange=lambda o, i: None) for r in range(P)]
        for s in doms:
            s.set_state(U)
        ms = [0.0] * P

        def timed(r, fn):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            fn()
            e1.record(st)
            return (e0, e1, r)

        def copy(attr_s, attr_r, nf):
            for q in range(P):
                for r in range(P):
                    b = doms[0].block
                    for f in range(nf):
                        getattr(doms[q], attr_r)[f, r * b:(r + 1) * b].copy_(getattr(doms[r], attr_s)[f, q * b:(q + 1) * b])

        evs = []
        for k in range(steps + 1):  # the first step is a warm-up
            bufs = [(s.U_hat, s._u0) for s in doms]
            for s in doms:
                s._umax.zero_()
            for rk in range(3):
                for r, (s, (A, B)) in enumerate(zip(doms, bufs)):
                    cur = A if rk == 0 else B
                    if s._primed != (cur.data_ptr(), cur._version):
                        evs.append(timed(r, lambda s=s, cur=cur: s.plan.slab_prime(cur)))
                copy("send1", "recv1", doms[0].n1)
                for r, s in enumerate(doms):
                    evs.append(timed(r, lambda s=s, rk=rk: s.plan.slab_middle(s._umax if rk == 0 else None)))
                copy("send2", "recv2", doms[0].n2)
                for r, (s, (A, B)) in enumerate(zip(doms, bufs)):
                    cur = A if rk == 0 else B
                    evs.append(timed(r, lambda s=s, rk=rk, cur=cur, A=A, B=B:
                                     s.plan.slab_stage(rk, s.dt, cur, A, None, B, None, 0)))
                    s._primed = (B.data_ptr(), B._version)
            for s, (A, B) in zip(doms, bufs):
                s.U_hat, s._u0 = B, A
                s._primed = (B.data_ptr(), B._version)
            if k == 0:
                torch.cuda.synchronize()
                evs = []
        torch.cuda.synchronize()
        for e0, e1, r in evs:
            ms[r] += e0.elapsed_time(e1)
        for s in doms:
            s.check()
        esz = 8
        sent = 3 * (doms[0].n1 + doms[0].n2) * (P - 1) * doms[0].block * esz  # bytes per rank per step
        comp = max(ms) / steps
        proj = comp + sent / 770e9 * 1e3
        out["P%d" % P] = {"per_rank_compute_ms_per_step": [round(m / steps, 3) for m in ms],
                          "compute_efficiency_vs_whole_grid": round(whole / steps * 1e3 / (P * comp), 3),
                          "exchange_bytes_per_rank_per_step": sent,
                          "model_exchange_ms_at_770GBs": round(sent / 770e9 * 1e3, 3),
                          "model_step_ms_no_overlap": round(proj, 3),
                          "model_value_no_overlap": round(float(n) ** 3 / (proj * 1e-3) / 1e6, 1)}
        del doms
        torch.cuda.empty_cache()
    out["unit"] = UNIT
    out["note"] = ("ranks emulated one after another on one GPU; the exchange time is modelled from the bytes, "
                   "not measured")
    return out


def bench_ensemble(rank, steps=200):
    """The 48-member ensemble: one captured graph per PERIOD steps (each member
    a stream branch) against the same members stepped one at a time."""
    import torch
    from sles.graph import Ensemble
    a, b = ensemble_members(rank), ensemble_members(rank)
    pts = sum(float(d.N) ** d.dim for d in a)
    ens = Ensemble(a)
    ens.advance(4)  # capture
    seq = Ensemble(b)
    seq.advance_sequential(4)
    st = torch.cuda.current_stream()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    e[0].record(st)
    ens.advance(steps)
    e[1].record(st)
    seq.advance_sequential(steps)
    e[2].record(st)
    torch.cuda.synchronize()
    tg, ts = e[0].elapsed_time(e[1]) / 1e3, e[1].elapsed_time(e[2]) / 1e3
    diffs = [rel_l2(x.U_hat, y.U_hat) for x, y in zip(a, b)]
    out = {"value": round(pts * steps / tg / 1e6, 2), "unit": UNIT, "members": len(a), "steps": steps,
           "points_per_step": pts, "sequential_value": round(pts * steps / ts / 1e6, 2),
           "speedup_vs_sequential": round(ts / tg, 3), "max_member_rel_l2_vs_sequential": max(diffs),
           "batches": [len(mb.members) for mb in ens.batches], "single_members": len(ens.units) - len(ens.batches),
           "config": "32 2D vorticity (N in {256,512,1024}, RK4) + 16 3D Smagorinsky (N in {64,96,128}, RK4), FP32; "
                     "members of one grid and scheme batched into one plan (one launch per pass, per-member nu and "
                     "Cs), batches and single members as branches of one replayed graph, vs members one at a time"}
    del a, b, ens, seq
    torch.cuda.empty_cache()
    return out


def bench_zoo(rank):
    """One short run of every kind of kernel the library launches (for an ncu
    capture of each kernel's first launch): the 3D fused passes at 256^3 FP32
    (Smagorinsky RK3 on every x variant, Vreman corrected ETD2, no-LES RK4,
    the alternative y/z variants), the FP64 passes, the 2D passes at 1024^2,
    the standalone transforms and diagnostics, the device-dt controller, the
    adjoint passes at 64^3 and 128^3 (direct-load and TMA-ring x passes), a
    slab decomposition and a member batch."""
    import torch
    from sles import ETD2_method, RK3_method, RK4_method, diagnostics
    from sles import _native as nat
    from sles.adjoint import RK4Rollout
    from sles.graph import MemberBatch
    from sles.initial import initial_vorticity
    from sles.initialize_domain import InitializeDomain
    from sles.slab import SlabDomain, emulated_exchange
    from sles.synthetic import gaussian_vorticity_2d
    done = []

    def release():
        torch.cuda.synchronize()
        torch.cuda.empty_cache()

    d = make_domain(256, "float32", rank)
    for v in range(4):
        d._plan.set_variant(v, nat.PASS_X)
        RK3_method.solveForNextTimestep(d)
    d._plan.set_variant(3, nat.PASS_X)
    for py, pz in ((1, 0), (0, 1)):
        d._plan.set_variant(py, nat.PASS_Y)
        d._plan.set_variant(pz, nat.PASS_Z)
        RK3_method.solveForNextTimestep(d)
    diagnostics.diag(d, with_max=True, nshell=200)
    U = d.U
    del d, U
    release()
    done.append("256^3 f32 smag rk3 (x variants 0-3, y/z variants), diag, c2r")
    d = make_domain(256, "float32", rank, method="ETD2", les="vreman", nu=5e-5, cs=math.sqrt(0.028), dt=5e-4,
                    k0=6.0, parity=False)
    for _ in range(2):
        ETD2_method.solveForNextTimestep(d)
    del d
    release()
    d = make_domain(256, "float32", rank, method="RK4", les=None)
    d.U_hat1[...] = d.U_hat
    RK4_method.solveForNextTimestep(d)
    del d
    release()
    d = make_domain(128, "float64", rank)
    RK3_method.solveForNextTimestep(d)
    del d
    release()
    done.append("256^3 vreman etd2, 256^3 no-LES rk4, 128^3 f64")
    for les in (None, "Smagorinsky"):
        d2 = InitializeDomain(nu=1e-4, dimension=2, time_stepSize=1e-3, No_of_gridpoint=(4 if les else 1) * 1024,
                              method="RK4", LES_ON=1 if les else 0, LES_model=les, Cs=0.17, dtype="float32")
        initial_vorticity(d2, gaussian_vorticity_2d(1024, seed=rank))
        d2.U_hat1[...] = d2.U_hat
        RK4_method.solveForNextTimestep(d2)
        del d2
        release()
    done.append("2D 1024^2 rk4 (no LES, Smagorinsky)")
    from sles.SM_solver import spectralMethodSolver
    import tempfile
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as td:
        os.chdir(td)
        try:
            d = make_domain(64, "float32", rank)
            d.T = 0.02
            spectralMethodSolver(d, No_Ek_plot=1, verbose=False, device_dt=True, chunk=4)
        finally:
            os.chdir(cwd)
    del d
    release()
    done.append("device-dt controller at 64^3")
    for na in (64, 128):  # direct-load adjoint x pass at 64^3, the TMA-ring one at 128^3
        ro = RK4Rollout(na, 1e-3, 1e-3, les="Smagorinsky", Cs=0.17, dtype=torch.float32, checkpoint_every=2)
        U0 = make_domain(na, "float32", rank, method="RK4").U_hat.clone().to(ro.cdtype)
        UT, ck = ro.forward_states(U0, 0.17, 2)
        ro.backward_states(ck, UT[..., : ro.nk].clone(), 0.17, 2)
        del ro, U0, UT, ck
        release()
        done.append("adjoint rk4 at %d^3" % na)
    base = make_domain(256, "float32", rank)
    doms = [SlabDomain(256, nu=NU, dt=DT, method="RK3", les="Smagorinsky", Cs=CS, dtype=torch.float32, nranks=2,
                       rank=r, exchange=lambda o, i: None) for r in range(2)]
    for sd in doms:
        sd.set_state(base.U_hat)
    emulated_exchange(doms)()
    del doms, base
    release()
    done.append("slab P=2 at 256^3")
    ms = [make_domain(128, "float32", rank + i, method="RK4", cs=0.12 + 0.02 * i) for i in range(3)]
    for m in ms:
        m.U_hat1[...] = m.U_hat
    mb = MemberBatch(ms)
    mb.step()
    del mb, ms
    release()
    done.append("member batch of 3 at 128^3")
    return {"ran": done}


def bench_kernels(case, n, precision, rank, xvar=-1):
    """Mean ms per launch of each kernel class of one RHS evaluation
    (sles_profile_rhs, CUDA events, 20 evaluations) and its algorithmic GB/s."""
    from sles import ETD2_method
    d = bench_case_domain(case, n, precision, rank)
    if xvar >= 0:
        d._plan.set_variant(xvar)
    kms = d._plan.profile_rhs(d._s_uhat, d._new_hc(3), 20)
    names = ["x_inverse", "y_inverse", "z_fused", "y_forward", "x_forward_combine"]
    les = case != "none"
    nf = (9, 15, 18, 15, 18) if les else (5, 8, 9, 6, 8)
    fbytes = float(n) * n * (n // 2 + 1) * (8 if precision == "float32" else 16)
    return {"case": case, "n": n, "precision": precision, "x_variant": d._plan.get_variant(0),
            "kernel_ms": {k: round(t, 4) for k, t in zip(names, kms)},
            "kernel_gbs": {k: round(b * fbytes / (t * 1e-3) / 1e9, 1) for k, b, t in zip(names, nf, kms)}}


def bench_case_domain(case, n, precision, rank):
    if case == "vreman_etd2":
        return make_domain(n, precision, rank, method="ETD2", les="vreman", nu=5e-5, cs=math.sqrt(0.07 / 2.5),
                           dt=5e-4, k0=6.0, parity=False)
    if case == "smag_rk4":
        d = make_domain(n, precision, rank, method="RK4")
        d.U_hat1[...] = d.U_hat
        return d
    return make_domain(n, precision, rank)


def bench_steps(case, n, precision, steps, warmup, rank, xvar=-1):
    """A plain stepping run of one workload (for ncu launch lists and
    captures): the Smagorinsky recipe with the reference RK3 or RK4, or the
    Vreman case with the corrected ETD2, at n^3."""
    from sles import ETD2_method, RK3_method, RK4_method
    if case == "vreman_etd2":
        d = make_domain(n, precision, rank, method="ETD2", les="vreman", nu=5e-5, cs=math.sqrt(0.07 / 2.5), dt=5e-4,
                        k0=6.0, parity=False)
        step = ETD2_method.solveForNextTimestep
    elif case == "smag_rk4":
        d = make_domain(n, precision, rank, method="RK4")
        d.U_hat1[...] = d.U_hat
        step = RK4_method.solveForNextTimestep
    else:
        d = make_domain(n, precision, rank)
        step = RK3_method.solveForNextTimestep
    if xvar >= 0:
        d._plan.set_variant(xvar)
    for _ in range(warmup):
        step(d)
    secs = time_steps(d, steps, step)
    d._plan.check()
    return {"case": case, "n": n, "precision": precision, "steps": steps, "ms_per_step": round(secs / steps * 1e3, 4),
            "x_variant": d._plan.get_variant(0)}


def headline_summary(out):
    """The headline figures in a few hundred characters (printed last)."""
    r = lambda x, k=4: None if x is None else (round(x, k) if isinstance(x, float) else x)
    ns = {"fp32_256": out["value"], "roofline_frac": out["roofline"]["frac"],
          "step_model_frac": out["step_roofline"]["frac"], "e2e_256": out["e2e"]["value"]}
    if "fp64" in out:
        f = out["fp64"]
        ns.update(fp64_fused_256=f["fused_fp64_value"], fp64_torch_256=f["torch_fft_fp64_value"],
                  fp32_vs_fp64_rel_l2=r(f["rel_l2_fp32_vs_fp64"], 10),
                  fp64_fused_vs_cpu_fp64=f.get("fused_fp64_vs_cpu_fp64"))
    if "n512" in out:
        a, b = out["n512"]["smagorinsky_rk3"], out["n512"]["vreman_etd2"]
        ns["n512_smag_rk3"] = {"value": a["value"], "x_torch_fp64": a["speedup_vs_torch_fp64"],
                               "rel_l2_100": r(a["rel_l2_fp32_vs_fp64_after_100_steps"], 10),
                               "ek_err_100": r(a["ek_err_fp32_vs_fp64_after_100_steps"][
                                   "max_rel_shells_above_1e-8_of_peak"], 8),
                               "step_model_frac": a["step_roofline_frac"], "kernel_gbs": a.get("kernel_gbs")}
        ns["n512_vreman_etd2"] = {"value": b["value"], "rel_l2_100": r(b["rel_l2_fp32_vs_fp64_after_100_steps"], 10),
                                  "step_model_frac": b["step_roofline_frac"]}
    if "cfg2_error_history" in out:
        h = out["cfg2_error_history"]
        ns["cfg2_500_steps"] = {"rel_l2_max": r(h["rel_l2_max"], 10), "ek_err_max": r(h["ek_err_max"], 8)}
    if "adjoint" in out:
        ns["adjoint_fwd_ratio"] = out["adjoint"]["adjoint_fwd_ratio"]
        ns["adjoint_cs_rel_err"] = r(out["adjoint"]["cs_rel_err_f64_vs_richardson"], 12)
    if "ensemble" in out:
        ns["ensemble_x_seq"] = out["ensemble"]["speedup_vs_sequential"]
    if "slab" in out:
        ns["slab512_compute_eff"] = {k: v["compute_efficiency_vs_whole_grid"] for k, v in out["slab"].items()
                                     if isinstance(v, dict)}
    if "fft_vs_cufft" in out:
        ns["fft_r2c_x_cufft"] = {k: v["speedup_r2c_vs_cufft"] for k, v in out["fft_vs_cufft"].items()
                                 if isinstance(v, dict)}
    return ns


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="sles", choices=["sles", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64 comparison runs")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the autotuner (use the default or cached kernel variants)")
    ap.add_argument("--only", choices=["n512", "adjoint", "ensemble", "driver", "fft", "steps", "kernels", "zoo", "slab",
                                       "cfg2"],
                    help="run one extra block alone and print it (profiling; not a bench line); 'steps': "
                         "--case at --n stepped --steps times after --warmup (for ncu launch lists)")
    ap.add_argument("--case", default="smag_rk3", choices=["smag_rk3", "vreman_etd2", "smag_rk4"],
                    help="workload of --only steps")
    ap.add_argument("--precision", default="float32", choices=["float32", "float64"])
    ap.add_argument("--xvar", type=int, default=-1, help="x-pass variant of --only steps (-1: default/cached)")
    args = ap.parse_args()
    assert args.warmup >= 3 or args.impl == "reference" or args.only, "at least 3 warm-up steps"
    global TUNE
    TUNE = not args.no_tune

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    from sles import RK3_method
    from sles import _stepper
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        return max_over_ranks_of(x, world, "cuda")

    n = args.n
    npts = float(n) ** 3
    step = RK3_method.solveForNextTimestep
    if args.only:
        peak, _ = measured_peak()
        fn = {"n512": lambda: bench_512(peak, rank), "adjoint": lambda: bench_adjoint(rank),
              "slab": lambda: bench_slab(rank),
              "ensemble": lambda: bench_ensemble(rank), "driver": lambda: bench_driver(rank),
              "fft": lambda: bench_fft(rank),
              "kernels": lambda: bench_kernels(args.case, args.n, args.precision, rank, args.xvar),
              "zoo": lambda: bench_zoo(rank),
              "cfg2": lambda: bench_cfg2_history(rank),
              "steps": lambda: bench_steps(args.case, args.n, args.precision, args.steps, args.warmup, rank,
                                           args.xvar)}[args.only]
        print(json.dumps({"only": args.only, "result": fn()}))
        return

    # ---------------- device-resident FP32 run (value) ----------------
    d = make_domain(n, "float32", seed=rank)
    tuned = tune_domain(d)
    for _ in range(args.warmup):
        step(d)
    _stepper.LAUNCHES[0] = 0
    barrier()
    with ClockSampler(gpu_index()) as clk:
        secs = time_steps(d, args.steps, step)
    launches = _stepper.LAUNCHES[0]
    d._plan.check()  # no bounded wait gave up during the timed steps
    value, secs = replicas_value(npts, args.steps, secs, world, "cuda")
    ms_step = secs / args.steps * 1e3

    # per-kernel times (CUDA events, same stream) for the roofline
    du = d._new_hc(3)
    kms = d._plan.profile_rhs(d._s_uhat, du, 20)
    del du
    names = ["x_inverse", "y_inverse", "z_fused", "y_forward", "x_forward_combine"]
    kdict = dict(zip(names, [round(x, 4) for x in kms]))
    peak, peak_src = measured_peak()
    fbytes = float(n) * n * (n // 2 + 1) * 8  # one half-complex FP32 field
    # the dominant kernel of the RHS evaluation timed above: algorithmic bytes
    # = half-complex fields read + written per launch
    rinfo = {"z_fused": (18, "k_zpass_f32_%d_smag" % n,
                         "k_zpass (fused z pass: c2r x12, u x omega, Smagorinsky stress, r2c x9)"),
             "x_forward_combine": (18, "k_xpass_f32_%d_smag_rhs_xv%d" % (n, d._plan.get_variant(0)),
                                   "k_xpass (x forward of 6 slots, kx stress part, mask, projection, viscous "
                                   "term, update, x inverse priming the next RHS; 9 fields in, 9 out)")}
    dom = max(rinfo, key=lambda k: kms[names.index(k)])
    nf_dom, tkey, kdesc = rinfo[dom]
    z_alg = nf_dom * fbytes
    z_ach = z_alg / (kms[names.index(dom)] * 1e-3) / 1e9
    traffic = ncu_traffic(tkey)
    step_alg = STEP_BYTES_PER_PT_RHS["f32"] * 3 * npts
    step_ach = step_alg / (ms_step * 1e-3) / 1e9

    # ---------------- end to end through the public API with host buffers ----------------
    # every step: its state copied in from pinned host memory, one RK3 step,
    # the result copied back to pinned host memory (sles.pipeline.HostStepper
    # overlaps step k's copies with its neighbours' compute on two copy streams)
    from sles.pipeline import HostStepper
    host_in = torch.empty(tuple(d.U_hat.shape), dtype=d.U_hat.dtype, pin_memory=True)
    host_out = torch.empty_like(host_in, pin_memory=True)
    host_in.copy_(d.U_hat)
    torch.cuda.synchronize()
    ke = max(40, args.steps)
    hs = HostStepper(d, steps=1)
    hs.run(host_in, [host_out] * 2)
    hs.synchronize()
    barrier()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    hs.run(host_in, [host_out] * ke)
    st.wait_stream(hs.d2h)  # the last device->host copy is inside the timed region
    e1.record(st)
    torch.cuda.synchronize()
    e2e_secs = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    e2e_value = world * npts * ke / e2e_secs / 1e6
    io_bytes = host_in.numel() * host_in.element_size()
    # the same per-step copies alone, both directions at once on the two copy
    # streams (no compute): the host-link bound of e2e
    hs.h2d.wait_stream(st)
    hs.d2h.wait_stream(st)
    torch.cuda.synchronize()
    e0.record(st)
    hs.h2d.wait_event(e0)
    hs.d2h.wait_event(e0)
    for k in range(ke):
        with torch.cuda.stream(hs.h2d):
            hs.din[k % 2].copy_(host_in, non_blocking=True)
        with torch.cuda.stream(hs.d2h):
            host_out.copy_(hs.dout[k % 2], non_blocking=True)
    st.wait_stream(hs.h2d)
    st.wait_stream(hs.d2h)
    e1.record(st)
    torch.cuda.synchronize()
    copy_secs = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    del host_in, host_out, hs

    out = {"metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded random-phase spectrum, seed=rank)",
           "config": bench_config(n, world),
           "precision": "fp32 fields/FFTs, fp64 twiddles", "autotune": tuned,
           "e2e": {"value": round(e2e_value, 2), "unit": UNIT, "h2d_bytes_per_step": io_bytes,
                   "d2h_bytes_per_step": io_bytes, "steps": ke,
                   "copies_only_value": round(world * npts * ke / copy_secs / 1e6, 2),
                   "copies_only_gbs_per_direction": round(io_bytes * ke / copy_secs / 1e9, 1),
                   "path": "sles.pipeline.HostStepper: per step pinned host -> U_hat, RK3_method."
                           "solveForNextTimestep, U_hat -> pinned host; copies on two streams overlap the "
                           "neighbouring steps' compute"},
           "gpu_launches": launches,
           "roofline": {"bound": "hbm", "kernel": kdesc,
                        "achieved": round(z_ach, 1), "peak": peak, "unit": "GB/s", "frac": round(z_ach / peak, 4),
                        "traffic": traffic, "algorithmic_bytes_per_launch": z_alg, "peak_source": peak_src},
           "step_roofline": {"model_bytes_per_step": step_alg, "achieved": round(step_ach, 1), "unit": "GB/s",
                             "frac": round(step_ach / peak, 4),
                             "model": "384 B/pt/RHS x 3 RHS/step (21 transforms x 16 B + 48 B state)"},
           "kernel_ms": kdict,
           "kernel_gbs": {k: round(b_ * fbytes / (kms[names.index(k)] * 1e-3) / 1e9, 1) for k, b_ in
                          (("x_inverse", 9), ("y_inverse", 15), ("z_fused", 18), ("y_forward", 15),
                           ("x_forward_combine", 18))}}

    # ---------------- FP64 comparisons ----------------
    if not args.no_compare:
        kc = min(args.steps, 20)
        d32 = make_domain(n, "float32", seed=rank)
        d64 = make_domain(n, "float64", seed=rank)
        for _ in range(2):
            step(d64)
            step(d32)
        s64 = time_steps(d64, kc, step)
        for _ in range(kc):
            step(d32)
        a, bref = d32.U_hat.to(torch.complex128), d64.U_hat
        err = float(torch.linalg.vector_norm(a - bref) / torch.linalg.vector_norm(bref))
        ek, klive, ekall = spectrum_error(a, bref, n)
        v64 = npts * kc / s64 / 1e6
        del d32, d64, a, bref
        torch.cuda.empty_cache()
        tp = torch_plain_fp64_rk3(n, 2, 1, rank)
        vtp = npts / tp / 1e6
        torch.cuda.empty_cache()
        out["fp64"] = {"fused_fp64_value": round(v64, 2), "torch_fft_fp64_value": round(vtp, 2),
                       "speedup_vs_fused_fp64": round(value / world / v64, 2),
                       "speedup_vs_torch_fp64": round(value / world / vtp, 2),
                       "rel_l2_fp32_vs_fp64": err, "steps_compared": kc + 2,
                       "ek_err_fp32_vs_fp64": {"max_rel_shells_above_1e-8_of_peak": ek, "up_to_shell": klive,
                                               "max_rel_all_shells": ekall},
                       "note": "FP32 fused vs FP64 fused (same kernels, float64) on the same seeded field"}
    if not args.no_compare and world == 1:
        out["cfg1_taylor_green"] = bench_cfg1(rank)
        out["cfg2_error_history"] = bench_cfg2_history(rank)
        out["fft_vs_cufft"] = bench_fft(rank)
        out["n512"] = bench_512(peak, rank)
        out["slab"] = bench_slab(rank)
        adj = bench_adjoint(rank)
        out["adjoint"] = adj
        out["adjoint_fwd_ratio"] = adj["adjoint_fwd_ratio"]
        out["ensemble"] = bench_ensemble(rank)
        out["driver_loop"] = bench_driver(rank)
    else:
        out["adjoint_fwd_ratio"] = None

    # ---------------- CPU baseline (oracle port, bounded sample) ----------------
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        cores = os.cpu_count() or 1
        v_cpu, secs_cpu = cpu_oracle_rate(n, 1, 0, 0, cores)
        out["cpu_baseline"] = {"value": round(v_cpu, 4), "unit": UNIT, "cores": cores, "kind": "port",
                               "sample": "1 RK3 step at %d^3 (%.1f s), NumPy + scipy.fft workers=%d" %
                                         (n, secs_cpu, cores)}
        if "fp64" in out:  # precision-matched: the fused float64 path against the float64 CPU port
            out["fp64"]["fused_fp64_vs_cpu_fp64"] = round(out["fp64"]["fused_fp64_value"] / v_cpu, 1)
    out["clocks"] = clk.summary()
    out["headline"] = headline_summary(out)  # last: the compact figures stay in a short stdout tail
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
