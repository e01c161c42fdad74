"""Host-resident states stepped through a domain with the copies overlapped.

The reference keeps its state in host memory; a caller that holds states on
the host (a batch of ensemble snapshots, a service answering requests) pays a
host->device copy before and a device->host copy after each advance.
``HostStepper`` hides them: item k's device->host copy and item k+1's
host->device copy run on their own streams while item k computes, through two
device staging buffers per direction.

    hs = HostStepper(domain, steps=1)
    hs.run(host_inputs, host_outputs)   # pinned (3, N, N, N//2+1) complex tensors
    hs.synchronize()

Each item starts from its host state (written into ``domain.U_hat``; U and
curl are derived from it, and an ETD2 domain restarts its bootstrap step) and
is advanced ``steps`` steps of the domain's scheme; its final ``U_hat`` lands
in the matching host output.  Outputs are complete after ``synchronize()``.
"""
from __future__ import annotations

import torch

from . import ETD2_method, RK3_method, RK4_method
from . import _native as nat

__all__ = ["HostStepper"]

_STEP = {"RK4": RK4_method.solveForNextTimestep, "RK3": RK3_method.solveForNextTimestep,
         "ETD2": ETD2_method.solveForNextTimestep}


class HostStepper:
    def __init__(self, domain, steps=1):
        self.d = domain
        self.steps = int(steps)
        shape, dt, dev = tuple(domain.U_hat.shape), domain.U_hat.dtype, domain.device
        self.din = [torch.empty(shape, dtype=dt, device=dev) for _ in range(2)]
        self.dout = [torch.empty(shape, dtype=dt, device=dev) for _ in range(2)]
        esz = torch.empty((), dtype=dt).element_size()
        # staging buffers [..][nk] <-> padded state [..][nkp]: rows copied by sles_copy_rows
        self._rowcopy = (domain._nk * esz, int(torch.Size(shape).numel()) // domain._nk, domain._nkp * esz)
        self.h2d = torch.cuda.Stream(dev)
        self.d2h = torch.cuda.Stream(dev)
        ev = lambda: [torch.cuda.Event() for _ in range(2)]
        self.in_ready, self.in_free, self.out_ready, self.out_free = ev(), ev(), ev(), ev()
        self._used = [False, False]
        self.bytes_in = self.bytes_out = 0

    def run(self, host_in, host_out):
        """Advance every item of ``host_in`` (a pinned tensor or a list of them;
        a single tensor with ``len(host_out)`` items reuses it) into ``host_out``."""
        d, cur = self.d, torch.cuda.current_stream(self.d.device)
        outs = host_out if isinstance(host_out, (list, tuple)) else [host_out]
        ins = host_in if isinstance(host_in, (list, tuple)) else [host_in] * len(outs)
        if len(ins) != len(outs):
            raise ValueError("host_in and host_out hold different numbers of items")
        step = _STEP[d.method]
        for k, (hi, ho) in enumerate(zip(ins, outs)):
            b = k % 2
            if self._used[b]:
                self.h2d.wait_event(self.in_free[b])   # the compute that read din[b] is done
            with torch.cuda.stream(self.h2d):
                self.din[b].copy_(hi, non_blocking=True)
                self.in_ready[b].record(self.h2d)
            cur.wait_event(self.in_ready[b])
            w, rows, pitch = self._rowcopy
            nat.copy_rows(d._s_uhat, self.din[b], w, rows, pitch, w, cur)
            if d.method in ("RK4", "ETD2"):            # RK4, or ETD2's RK4 bootstrap step:
                nat.copy_rows(d._s_u1, self.din[b], w, rows, pitch, w, cur)  # U_hat1 = U_hat (SM_solver.py:33)
            d._mark_stepped()                          # stage 0 derives U and curl from this U_hat
            d._primed = None                           # a raw copy: the workspace holds no x inverse of it
            if d.method == "ETD2":
                d.firstIteration = True                # each item starts its own ETD2 history
            self.in_free[b].record(cur)
            for _ in range(self.steps):
                step(d)
            if self._used[b]:
                cur.wait_event(self.out_free[b])      # the host copy of dout[b] is done
            nat.copy_rows(self.dout[b], d._s_uhat, w, rows, w, pitch, cur)
            self.out_ready[b].record(cur)
            self.d2h.wait_event(self.out_ready[b])
            with torch.cuda.stream(self.d2h):
                ho.copy_(self.dout[b], non_blocking=True)
                self.out_free[b].record(self.d2h)
            self._used[b] = True
            self.bytes_in += hi.numel() * hi.element_size()
            self.bytes_out += ho.numel() * ho.element_size()

    def synchronize(self):
        """Wait for every queued copy and step (host outputs complete)."""
        torch.cuda.current_stream(self.d.device).synchronize()
        self.d2h.synchronize()
        self.h2d.synchronize()
        self.d._plan.check()
