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
from . import _native as nat
from . import autotune

__all__ = ["CapturedStepper", "Ensemble", "MemberBatch", "PERIOD"]

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


class _DomainUnit:
    """One domain as a unit of a capture: steps through its own plan."""

    def __init__(self, d):
        self.d = d

    def step(self):
        _eager_step(self.d)

    def state_key(self):
        return _state_key(self.d)

    def stepped(self):
        self.d._mark_stepped()


class MemberBatch:
    """Ensemble members of one grid, dimension, precision, closure, scheme,
    parity, dt and forcing stepped as one: a batched plan
    (``sles_plan_set_batch``) runs each pass of every member in one launch,
    with each member's own viscosity and C_s.  The batch keeps the states in
    tensors laid out [component][member][...]; ``scatter`` writes them back
    into the members (the Ensemble does so after every ``advance``).  Every
    member's first step derives U and curl from its U_hat (a domain stepped
    alone reuses the physical fields its initial-condition setter stored, which
    agree to round-off)."""

    @staticmethod
    def key(d):
        return (d.dim, d.N, d._rdtype, d.LES_model, d.method, d.parity_mode, float(d.dt), float(d.forcing),
                str(d.device))

    def __init__(self, domains):
        self.members = list(domains)
        d0 = self.members[0]
        if any(MemberBatch.key(d) != MemberBatch.key(d0) for d in self.members):
            raise ValueError("a member batch needs one grid, dimension, precision, closure, scheme, parity, dt")
        if d0.method not in ("RK3", "RK4"):
            raise ValueError("member batches step RK3 or RK4")
        les = nat.LES_NONE
        if d0.LES_ON:
            les = nat.LES_SMAGORINSKY if d0.LES_model[0] == "S" else nat.LES_VREMAN
        scheme = nat.SCHEME_RK4 if d0.method == "RK4" else nat.SCHEME_RK3
        self.plan = nat.Plan(d0.dim, d0.N, d0._rdtype, les, scheme, d0.parity_mode, d0.nu, d0.Cs, d0.forcing,
                             d0.device, batch=([d.nu for d in self.members], [d.Cs for d in self.members]))
        autotune.apply_cached(self.plan, d0.method)
        self.method, self.dt = d0.method, float(d0.dt)
        shape = (d0.dim, len(self.members)) + tuple(d0._s_uhat.shape[1:])
        self.A = torch.empty(shape, dtype=d0._s_uhat.dtype, device=d0.device)
        self.B = torch.zeros_like(self.A)
        self.C = torch.empty_like(self.A) if self.method == "RK4" else None
        for b, d in enumerate(self.members):
            self.A[:, b].copy_(d._s_uhat)
            if self.C is not None:
                self.C[:, b].copy_(d._s_u1)
        self._primed = None

    def step(self):
        """One step of every member (src/RK4_method.py:20-35 / src/RK3_method.py:20-41)."""
        A, B, C = self.A, self.B, self.C
        nst = 4 if self.method == "RK4" else 3
        base = nat.STAGE_RK4 if self.method == "RK4" else 0
        for rk in range(nst):
            ucur = A if rk == 0 else B
            primed = rk > 0 or self._primed == A.data_ptr()
            self.plan.stage(rk, self.dt, ucur, A, C, B, None, None, None, base | (nat.STAGE_PRIMED if primed else 0))
        self.A, self.B = B, A
        self._primed = B.data_ptr()

    def state_key(self):
        return (self.A.data_ptr(), self.B.data_ptr(), self._primed)

    def stepped(self):
        pass

    def scatter(self):
        """Write the batch's states back into the member domains."""
        for b, d in enumerate(self.members):
            d._s_uhat.copy_(self.A[:, b])
            if self.C is not None:
                d._s_u1.copy_(self.C[:, b])
            d._mark_stepped()
            d._primed = None


class _Capture:
    """One CUDA graph advancing several units (domains or member batches) by
    PERIOD steps, each unit on its own captured stream (independent branches
    of the graph)."""

    def __init__(self, domains):
        self.domains = [u if isinstance(u, (MemberBatch, _DomainUnit)) else _DomainUnit(u) for u in domains]
        self.graph = None
        self.keys = None

    def valid(self):
        return self.graph is not None and [u.state_key() for u in self.domains] == self.keys

    def warm_and_capture(self):
        """Run PERIOD eager steps (first-step logic, cached launch attributes,
        primed workspaces), then record PERIOD steps.  Returns the number of
        steps executed on the GPU (PERIOD)."""
        self.graph = None
        for _ in range(PERIOD):
            for u in self.domains:
                u.step()
        torch.cuda.synchronize()
        before = [u.state_key() for u in self.domains]
        main = torch.cuda.Stream()
        side = [torch.cuda.Stream() for _ in self.domains]
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=main):
            # fork every branch from the graph's start before joining any, so
            # the members' launch sequences are independent (concurrent) nodes
            for s in side:
                s.wait_stream(main)
            for u, s in zip(self.domains, side):
                with torch.cuda.stream(s):
                    for _ in range(PERIOD):
                        u.step()
            for s in side:
                main.wait_stream(s)
        after = [u.state_key() for u in self.domains]
        if after != before:
            raise RuntimeError("step state did not return to its start after %d steps" % PERIOD)
        self.graph, self.keys = g, after
        return PERIOD

    def replay(self):
        self.graph.replay()
        for u in self.domains:
            u.stepped()


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
    together: one graph replay advances every member by PERIOD steps.  With
    ``batch=True`` (the default) members sharing a grid, dimension, precision,
    closure, RK scheme, parity, dt and forcing form a MemberBatch (one launch
    per pass for all of them, each with its own viscosity and C_s); every
    batch and every remaining member is a branch of the graph on its own
    captured stream, so they run concurrently."""

    def __init__(self, domains, batch=True):
        self.members = list(domains)
        self.batches = []
        units = []
        if batch:
            groups = {}
            for d in self.members:
                groups.setdefault(MemberBatch.key(d), []).append(d)
            for k, ds in groups.items():
                if len(ds) > 1 and ds[0].method in ("RK3", "RK4"):
                    mb = MemberBatch(ds)
                    self.batches.append(mb)
                    units.append(mb)
                else:
                    units.extend(_DomainUnit(d) for d in ds)
        else:
            units = [_DomainUnit(d) for d in self.members]
        self.units = units
        self._c = _Capture(units)

    def advance(self, nsteps):
        def one():
            for u in self.units:
                u.step()
        _advance(self._c, nsteps, one)
        for mb in self.batches:
            mb.scatter()

    def advance_sequential(self, nsteps):
        """The same steps run member by member without graphs (comparison)."""
        for d in self.members:
            for _ in range(int(nsteps)):
                _eager_step(d)
