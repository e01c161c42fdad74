"""Driver loop (src/SM_solver.py:18-83) with the reference's adaptive dt.

The loop, its CFL rule (dt = min(CFL dx/u_max, 0.1 dx^2/nu), with CFL = 0.3 on
the first step), the NaN stop and the "time per gridpoint per timestep" print
follow the reference.  Energy-spectrum snapshots go to Ek_plot_data.csv with
the reference's binning; field dumps (every ``file_out_time``) go to
dumpfile/ as raw float64 files with XDMF descriptions instead of HDF5 (h5py
is not used); the PNG plot is not produced (plotting is outside this library).
"""
from __future__ import annotations

import os
import time

import numpy as np

from . import ETD2_method as ETD2
from . import RK3_method as RK3
from . import RK4_method as RK4
from .diagnostics import max_velocity, reference_binned_spectrum
from .utilites import write_fields_xdmf

__all__ = ["spectralMethodSolver", "find_max_velocity", "compute_dt", "output_h5"]


def find_max_velocity(U, comm=None):
    """Signed max over all components and points (src/SM_solver.py:245-255)."""
    import torch
    if isinstance(U, torch.Tensor):
        return float(torch.max(U).item())
    return float(np.max(np.array([np.max(np.asarray(u)) for u in U])))


def compute_dt(U, u_max, nu, comm=None, dx=1.0, CFL=0.5):
    """src/SM_solver.py:258-277; raises SystemExit where the reference exits."""
    dt1 = CFL * dx / u_max
    dt2 = 0.1 * dx ** 2 / nu if (nu > 0) else 1e6
    dt = min(dt1, dt2)
    if dt < 1e-6:
        print(f"\n\n ###  Time step (dt = {dt:g}) is smaller than 1e-6  ###\n\n")
        raise SystemExit(1)
    return dt


def output_h5(domain, t, file_out_time, directory="dumpfile"):
    """Write the physical velocity (2D: u, v and the vorticity) at time t, as
    src/SM_solver.py:280-302 does, into ``directory``/dump{t//file_out_time}:
    raw float64 files with an XDMF description (utilites.write_fields_xdmf;
    h5py is not used)."""
    d = domain
    U = d.U.to("cpu").double().numpy()
    if d.dim == 2:
        fields = {"u": U[0], "v": U[1], "omega": d.curl.to("cpu").double().numpy()}
    else:
        fields = {"u": U[0], "v": U[1], "w": U[2]}
    os.makedirs(directory, exist_ok=True)
    return write_fields_xdmf(os.path.join(directory, f"dump{t // file_out_time:g}"), fields, d.dx, time=t)


def _step(domain):
    if domain.method == "RK4":
        RK4.solveForNextTimestep(domain)
    elif domain.method == "ETD2":
        ETD2.solveForNextTimestep(domain)
    elif domain.method == "RK3":
        RK3.solveForNextTimestep(domain)
    else:
        raise ValueError("Invalid method name")


def spectralMethodSolver(domain, file_out_time: float = 0.0, No_Ek_plot: int = 5, verbose: bool = True,
                         device_dt: bool = False, chunk: int = 32):
    """src/SM_solver.py:18-83.  device_dt=True runs the same loop with the
    time-step logic on the GPU (u_max reduced inside the fused z pass, dt and t
    kept in device memory) and the steps replayed as CUDA graphs of ``chunk``
    steps; the host synchronises once per chunk and at each E(k) snapshot,
    giving the same steps, dt sequence and snapshots as the host loop."""
    if device_dt:
        return _solver_device_dt(domain, file_out_time, No_Ek_plot, verbose, chunk)
    d = domain
    u_max = max_velocity(d)
    d.dt = compute_dt(None, u_max, d.nu, dx=d.dx, CFL=0.3)
    t = d.dt
    Ek_interval = d.T / No_Ek_plot if No_Ek_plot != 0 else 0
    Ek_counter = 0
    start = time.time()
    d.U_hat1[...] = d.U_hat            # src/SM_solver.py:33
    columns = {}
    counter = 0
    file_time = 0.0
    while True:
        if file_out_time > 0 and t >= file_time:     # src/SM_solver.py:40-42
            output_h5(d, t, file_out_time)
            file_time += file_out_time
        if Ek_interval > 0 and t >= Ek_counter:
            tk, tE = reference_binned_spectrum(d)
            columns[f"k-{t:g}"] = tk
            columns[f"Ek-{t:g}"] = tE
            Ek_counter += Ek_interval
        if (t >= d.T) or (d.dt < 1e-8):
            break
        t += d.dt
        _step(d)
        u_max = max_velocity(d)
        d.dt = compute_dt(None, u_max, d.nu, dx=d.dx, CFL=d.CFL)
        if d.dt != d.dt:
            if verbose:
                print("\n############ dt = Nan #############\n", counter)
            break
        counter += 1
    d._plan.check()  # a kernel's bounded wait that gave up raises here
    if columns:
        import pandas as pd
        pd.DataFrame(columns).to_csv("Ek_plot_data.csv", index=False)
    total = time.time() - start
    if verbose and counter > 0:
        print(f"=>  run time: {total} sec")
        print(f"Time per gridpoint per timestep: {total * d.num_processes / (d.N ** d.dim * counter)}\n")
    return counter


def _solver_device_dt(d, file_out_time, No_Ek_plot, verbose, chunk):
    import torch

    from . import _native as nat
    from .graph import CapturedStepper
    Ek_interval = d.T / No_Ek_plot if No_Ek_plot != 0 else 0
    c = nat.DtCtl()
    c.t_end, c.cfl_first, c.cfl, c.dx, c.nu = d.T, 0.3, d.CFL, d.dx, d.nu
    start = time.time()
    d.U_hat1[...] = d.U_hat            # src/SM_solver.py:33
    columns = {}
    Ek_counter = 0.0
    file_time = 0.0
    inf = float("inf")

    def events(t):
        """The loop's per-iteration outputs (src/SM_solver.py:40-45) due at t."""
        nonlocal Ek_counter, file_time
        if file_out_time > 0 and t >= file_time:
            output_h5(d, t, file_out_time)
            file_time += file_out_time
        if Ek_interval > 0 and t >= Ek_counter:
            tk, tE = reference_binned_spectrum(d)
            columns[f"k-{t:g}"] = tk
            columns[f"Ek-{t:g}"] = tE
            Ek_counter += Ek_interval
        # the controller pauses when t reaches the earlier of the next two
        return min(Ek_counter if Ek_interval > 0 else inf, file_time if file_out_time > 0 else inf)

    # the first iteration's outputs (t = dt_0 >= 0) are written here, so that
    # the first device step is never a paused one
    c.ek_next = events(compute_dt(None, max_velocity(d), d.nu, dx=d.dx, CFL=0.3))
    c.resumed = 1 if c.ek_next < inf else 0
    ctl = torch.frombuffer(bytearray(bytes(c)), dtype=torch.uint8).to(d.device)
    d._dtctl, d._parity = ctl, 0
    stepper = CapturedStepper(d)
    n_next = chunk
    try:
        while True:
            stepper.advance(n_next)
            st = nat.DtCtl.from_buffer_copy(bytes(ctl.cpu().numpy()))
            # next chunk: about the steps left before the next snapshot or the
            # end at the current dt (a chunk that overshoots runs paused no-op steps)
            nxt = min(st.ek_next, st.t_end) - st.t
            est = int(nxt / st.dt) + 1 if st.dt > 0 and nxt == nxt else chunk
            n_next = max(2, min(chunk, est))
            n_next += n_next % 2
            if st.flags & nat.DT_SNAPSHOT:
                st.ek_next = events(st.t)
                st.flags, st.paused, st.resumed = st.flags & ~nat.DT_SNAPSHOT, 0, 1
                ctl.copy_(torch.frombuffer(bytearray(bytes(st)), dtype=torch.uint8))
                continue
            if st.flags & nat.DT_NAN:
                if verbose:
                    print("\n############ dt = Nan #############\n", st.nsteps)
                break
            if st.flags & nat.DT_TOO_SMALL:
                print(f"\n\n ###  Time step (dt = {st.dt:g}) is smaller than 1e-6  ###\n\n")
                raise SystemExit(1)
            if st.flags & nat.DT_DONE:
                break
    finally:
        torch.cuda.synchronize(d.device)
        d._dtctl = None
    d.dt = st.dt
    counter = st.nsteps
    d._plan.check()  # a kernel's bounded wait that gave up raises here
    if columns:
        import pandas as pd
        pd.DataFrame(columns).to_csv("Ek_plot_data.csv", index=False)
    total = time.time() - start
    if verbose and counter > 0:
        print(f"=>  run time: {total} sec")
        print(f"Time per gridpoint per timestep: {total * d.num_processes / (d.N ** d.dim * counter)}\n")
    return counter
