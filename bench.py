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


def workload_name(n):
    return ("decaying isotropic turbulence LES %d^3, Smagorinsky Cs=%.2f (Delta=2pi/%d), reference RK3, "
            "dt=%g, nu=%g, random-phase spectrum k0=%g u0=%g" % (n, CS, n, DT, NU, K0, U0))


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
def make_domain(n, dtype, seed):
    import torch
    from sles.initialize_domain import InitializeDomain
    from sles.initial import initial_velocity
    from sles.synthetic import random_spectrum_velocity
    d = InitializeDomain(nu=NU, dimension=3, time_stepSize=DT, No_of_gridpoint=4 * n, method="RK3", LES_ON=1,
                         LES_model="Smagorinsky", Cs=CS, dtype=dtype)
    u, v, w = random_spectrum_velocity(n, K0, U0, seed=seed)
    initial_velocity(d, u, v, w)
    del u, v, w
    torch.cuda.synchronize()
    return d


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


def run_reference(args, rank, world):
    if rank != 0:
        return
    n = args.n
    cores = os.cpu_count() or 1
    w = min(args.warmup, 1)
    k = max(1, min(args.steps, 2))
    value, secs = cpu_oracle_rate(n, k, w, 0, cores)
    sample = ("%d timed RK3 step(s) at %d^3 after %d warm-up step(s) of the requested %d/%d; oracle port "
              "(NumPy + scipy.fft workers=%d) on the host cores" % (k, n, w, args.steps, args.warmup, cores))
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
           "steps": k, "warmup": w, "ms_per_step": round(secs / k * 1e3, 2), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, seed 0)",
           "config": {"workload": workload_name(n), "n": n, "scheme": "RK3 (reference)", "les": "Smagorinsky"},
           "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": cores, "kind": "port",
                            "sample": sample},
           "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="sles", choices=["sles", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64 comparison runs")
    args = ap.parse_args()
    assert args.warmup >= 3 or args.impl == "reference", "at least 3 warm-up steps"

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
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n = args.n
    npts = float(n) ** 3
    step = RK3_method.solveForNextTimestep

    # ---------------- device-resident FP32 run (value) ----------------
    d = make_domain(n, "float32", seed=rank)
    for _ in range(args.warmup):
        step(d)
    _stepper.LAUNCHES[0] = 0
    barrier()
    with ClockSampler(gpu_index()) as clk:
        secs = time_steps(d, args.steps, step)
    launches = _stepper.LAUNCHES[0]
    secs = max_over_ranks(secs)
    value = world * npts * args.steps / secs / 1e6
    ms_step = secs / args.steps * 1e3

    # per-kernel times (CUDA events, same stream) for the roofline
    du = d._new_hc(3)
    kms = d._plan.profile_rhs(d._s_uhat, du, 20)
    del du
    names = ["x_inverse", "y_inverse", "z_fused", "y_forward", "x_forward_combine"]
    kdict = dict(zip(names, [round(x, 4) for x in kms]))
    peak, peak_src = measured_peak()
    fbytes = float(n) * n * (n // 2 + 1) * 8  # one half-complex FP32 field
    z_alg = 18 * fbytes                         # z pass: 9 fields in, 9 out
    z_ach = z_alg / (kms[2] * 1e-3) / 1e9
    traffic = ncu_traffic("k_zpass_f32_%d_smag" % n)
    step_alg = STEP_BYTES_PER_PT_RHS["f32"] * 3 * npts
    step_ach = step_alg / (ms_step * 1e-3) / 1e9

    # ---------------- end to end through the public API with host buffers ----------------
    host_in = torch.empty(tuple(d.U_hat.shape), dtype=d.U_hat.dtype, pin_memory=True)
    host_out = torch.empty_like(host_in, pin_memory=True)
    host_in.copy_(d.U_hat)
    torch.cuda.synchronize()
    ke = max(10, args.steps // 4)

    def e2e_step(dd):
        dd.U_hat.copy_(host_in, non_blocking=True)
        step(dd)
        host_out.copy_(dd.U_hat, non_blocking=True)

    e2e_step(d)
    barrier()
    e2e_secs = max_over_ranks(time_steps(d, ke, e2e_step))
    e2e_value = world * npts * ke / e2e_secs / 1e6
    io_bytes = host_in.numel() * host_in.element_size()
    del host_in, host_out

    out = {"metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded random-phase spectrum, seed=rank)",
           "config": {"workload": workload_name(n), "n": n, "scheme": "RK3 (reference arithmetic)",
                      "les": "Smagorinsky", "precision": "fp32 fields/FFTs, fp64 twiddles",
                      "l2": "inputs larger than L2 (state 3x3x%.0f MB + workspace 9 fields)" % (fbytes / 1e6),
                      "parallelism": "replicas" if world > 1 else "single GPU"},
           "e2e": {"value": round(e2e_value, 2), "unit": UNIT, "h2d_bytes_per_step": io_bytes,
                   "d2h_bytes_per_step": io_bytes, "steps": ke,
                   "path": "domain.U_hat <- pinned host; RK3_method.solveForNextTimestep; pinned host <- U_hat"},
           "gpu_launches": launches,
           "roofline": {"bound": "hbm", "kernel": "k_zpass (fused z pass: c2r x12, u x omega, Smagorinsky "
                                                  "stress, r2c x9)",
                        "achieved": round(z_ach, 1), "peak": peak, "unit": "GB/s", "frac": round(z_ach / peak, 4),
                        "traffic": traffic, "algorithmic_bytes_per_launch": z_alg, "peak_source": peak_src},
           "step_roofline": {"model_bytes_per_step": step_alg, "achieved": round(step_ach, 1), "unit": "GB/s",
                             "frac": round(step_ach / peak, 4),
                             "model": "384 B/pt/RHS x 3 RHS/step (21 transforms x 16 B + 48 B state)"},
           "kernel_ms": kdict}

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
                       "note": "FP32 fused vs FP64 fused (same kernels, float64) on the same seeded field"}
    out["adjoint_fwd_ratio"] = None

    # ---------------- CPU baseline (oracle port, bounded sample) ----------------
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        cores = os.cpu_count() or 1
        v_cpu, secs_cpu = cpu_oracle_rate(n, 1, 0, 0, cores)
        out["cpu_baseline"] = {"value": round(v_cpu, 4), "unit": UNIT, "cores": cores, "kind": "port",
                               "sample": "1 RK3 step at %d^3 (%.1f s), NumPy + scipy.fft workers=%d" %
                                         (n, secs_cpu, cores)}
    out["clocks"] = clk.summary()
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
