"""Time the reference's own CPU code beside the oracle port (test
infrastructure: a calibration of the CPU baseline, never the product).

The reference (a-k-sangwan/spectral-LES) needs mpi4py and mpi4py-fft, which
this image lacks, so it runs here under the single-rank shim of
tests/golden/make_golden.py, with the shim's PFFT backed by scipy.fft using
``--workers`` threads (the reference's own arithmetic, FFTs threaded as
FFTW would be under one MPI rank).  The same RK3 Smagorinsky step at the
bench workload (random-phase spectrum k0=4, u0=1, nu=1e-4, Cs=0.17, dt=1e-3)
is then timed with the oracle port (oracle/spectral_oracle.py, scipy.fft
with the same workers).  Prints one JSON line: seconds per step of each and
their ratio, which converts the bench's port-based CPU baseline into
reference terms.

    python oracle/time_reference.py --reference <path of a reference checkout> [--n 256] [--workers 8]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--workers", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--steps", type=int, default=1)
    a = ap.parse_args(argv)
    sys.path.insert(0, os.path.join(REPO, "tests", "golden"))
    sys.path.insert(0, REPO)
    import make_golden as mg
    import scipy.fft as sfft
    mg.REF = a.reference
    ref = mg.import_reference()
    PFFT = sys.modules["mpi4py_fft"].PFFT

    def forward(self, x, out=None, normalize=False):  # the shim's PFFT on scipy.fft threads
        r = sfft.rfftn(np.asarray(x), axes=self.axes, workers=a.workers)
        if normalize:
            r = r / self.ntot
        if out is not None:
            out[...] = r
            return out
        return r

    def backward(self, x, out=None, normalize=True):
        r = sfft.irfftn(np.asarray(x), s=self.shape, axes=self.axes, workers=a.workers)
        if not normalize:
            r = r * self.ntot
        if out is not None:
            out[...] = r
            return out
        return r
    PFFT.forward, PFFT.backward = forward, backward

    from oracle import spectral_oracle as so
    n = a.n
    u = so.random_spectrum_velocity(n, k0=4.0, u0=1.0, seed=0)
    d = ref["initialize_domain"].InitializeDomain(nu=1e-4, dimension=3, time_stepSize=1e-3, No_of_gridpoint=4 * n,
                                                  method="RK3", LES_ON=1, LES_model="Smagorinsky", Cs=0.17)
    ref["initial"].initial_velocity(d, *u)
    d.U_hat1[:] = d.U_hat
    ref["RK3_method"].solveForNextTimestep(d)  # warm-up
    t0 = time.perf_counter()
    for _ in range(a.steps):
        ref["RK3_method"].solveForNextTimestep(d)
    t_ref = (time.perf_counter() - t0) / a.steps
    so.set_fft_workers(a.workers)
    o = so.OracleDomain(n, 3, nu=1e-4, dt=1e-3, les_model="Smagorinsky", Cs=0.17, method="RK3")
    so.initial_velocity(o, *u)
    so.step(o)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        so.step(o)
    t_port = (time.perf_counter() - t0) / a.steps
    print(json.dumps({"n": n, "workers": a.workers, "cores": os.cpu_count(), "reference_s_per_step": round(t_ref, 3),
                      "port_s_per_step": round(t_port, 3), "reference_over_port": round(t_ref / t_port, 3),
                      "reference_mpts_steps_s": round(n ** 3 / t_ref / 1e6, 4),
                      "port_mpts_steps_s": round(n ** 3 / t_port / 1e6, 4)}))


if __name__ == "__main__":
    main()
