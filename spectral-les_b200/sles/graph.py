"""CUDA-graph replay of time steps, and ensembles of domains stepped together.

A step is a fixed sequence of kernel launches on the current stream (no host
synchronization, no allocation), so it can be captured once and replayed.
The steppers swap buffer roles instead of copying (U_hat <-> U_hat0 each RK
step, F0 <-> F1 each ETD2 step); after two steps every role is back where it
started, so a capture of ``PERIOD`` steps replays consistently.

A capture is taken lazily by ``advance``: the first ``PERIOD`` steps of a
capture cycle run eagerly (they count toward the requested steps), the next
``PERIOD`` steps are recorded, and every later ``PERIOD`` steps are one
replay.  dt, nu, Cs and the forcing are baked into the captured launches; a
change to any of them, an in-place write to ``U_hat`` or reading ``U``/``curl``
(which reuses the workspace) makes the next ``advance`` capture again.
"""
from __future__ import annotations

import torch

from . import ETD2_method, RK3_method, RK4_method

__all__ = ["CapturedStepper", "Ensemble", "PERIOD"]

PERIOD = 2
_STEP = {"RK4": RK4_method.solveForNextTimestep, "RK3": RK3_method.solveForNextTimestep,
         "ETD2": ETD2_method.solveForNextTimestep}


def _eager_step(d):
    _STEP[d.method](d)


def _state_key(d):
    """Buffer roles, workspace priming and baked-in parameters of a domain."""
    roles = tuple(None if s is None else s.data_ptr() for s in (d._s_uhat, d._s_u0, d._s_u1, d._s_f0, d._s_f1))
    ctl = None if d._dtctl is None else d._dtctl.data_ptr()
    return roles, d._primed, (d.dt, d.nu, d.Cs, d.forcing), d.firstIteration, ctl, d._parity


class _Capture:
    """One CUDA graph advancing several domains by PERIOD steps, each domain
    on its own captured stream (independent branches of the graph)."""

    def __init__(self, domains):
        self.domains = list(domains)
        self.graph = None
        self.keys = None

    def valid(self):
        return self.graph is not None and [_state_key(d) for d in self.domains] == self.keys

    def warm_and_capture(self):
        """Run PERIOD eager steps (first-step logic, cached launch attributes,
        primed workspaces), then record PERIOD steps.  Returns the number of
        steps executed on the GPU (PERIOD)."""
        self.graph = None
        for _ in range(PERIOD):
            for d in self.domains:
                _eager_step(d)
        torch.cuda.synchronize()
        before = [_state_key(d) for d in self.domains]
        main = torch.cuda.Stream()
        side = [torch.cuda.Stream() for _ in self.domains]
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=main):
            # fork every branch from the graph's start before joining any, so
            # the members' launch sequences are independent (concurrent) nodes
            for s in side:
                s.wait_stream(main)
            for d, s in zip(self.domains, side):
                with torch.cuda.stream(s):
                    for _ in range(PERIOD):
                        _eager_step(d)
            for s in side:
                main.wait_stream(s)
        after = [_state_key(d) for d in self.domains]
        if after != before:
            raise RuntimeError("step state did not return to its start after %d steps" % PERIOD)
        self.graph, self.keys = g, after
        return PERIOD

    def replay(self):
        self.graph.replay()
        for d in self.domains:
            d._mark_stepped()


def _advance(cap, nsteps, eager_one):
    n = int(nsteps)
    while n >= 2 * PERIOD or (n >= PERIOD and cap.valid()):
        if not cap.valid():
            n -= cap.warm_and_capture()
            continue
        cap.replay()
        n -= PERIOD
    for _ in range(n):
        eager_one()


class CapturedStepper:
    """Advance one domain by whole steps through a replayed CUDA graph.

        cs = CapturedStepper(domain)
        cs.advance(200)   # 2 eager steps, then replays of a 2-step graph
    """

    def __init__(self, domain):
        self.domain = domain
        self._c = _Capture([domain])

    def advance(self, nsteps):
        _advance(self._c, nsteps, lambda: _eager_step(self.domain))


class Ensemble:
    """Independent domains of any grid size, dimension and parameters, stepped
    together: one graph replay advances every member by PERIOD steps, each
    member on its own captured stream so small members run concurrently."""

    def __init__(self, domains):
        self.members = list(domains)
        self._c = _Capture(self.members)

    def advance(self, nsteps):
        def one():
            for d in self.members:
                _eager_step(d)
        _advance(self._c, nsteps, one)

    def advance_sequential(self, nsteps):
        """The same steps run member by member without graphs (comparison)."""
        for d in self.members:
            for _ in range(int(nsteps)):
                _eager_step(d)
