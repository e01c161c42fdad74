"""Differentiable RK4 and RK3 rollouts: the fused forward steps with a
hand-written discrete adjoint behind ``torch.autograd.Function`` (3D).

    ro = RK4Rollout(n=128, nu=2e-4, dt=2e-3, les="Smagorinsky", dtype=torch.float32,
                    checkpoint_every=10)
    U0 = ro.rfft(u_phys).requires_grad_()          # (3, n, n, n//2+1) complex
    Cs = torch.tensor(0.17, dtype=torch.float64, requires_grad=True)
    UT = ro(U0, Cs, nsteps=100)                    # fused RK4 steps (src/RK4_method.py:20-71)
    loss = log_spectrum_misfit(UT, E_target, n)
    loss.backward()                                # U0.grad, Cs.grad

The forward keeps the state every ``checkpoint_every`` steps.  The backward
walks the segments from the last to the first: it recomputes a segment's
steps from its checkpoint, keeping each step's four stage states, then runs
the reverse stages (``sles_adjoint_stage``, the transpose of the fused
right-hand side and of the step's stage combination) through it.  Gradients
follow torch's convention for complex tensors (dL/dRe + i dL/dIm of every
stored half-complex entry), so they compare directly with torch.fft autograd.

``RK3Rollout`` is the same for the reference's RK3 (src/RK3_method.py:20-41,
whose stages are U_0 + dt/2 k_0, U_0 + dt k_1 and the output U_0 + dt k_2)
or, with ``parity=False``, for the corrected SSP-RK3 (Shu & Osher 1988).
``ETD2Rollout`` is the corrected ETD2 (Cox & Matthews 2002) with the
reference's step structure (src/ETD2_method.py:7-57: the first step records
F(U_0) and runs RK4); the reference's own ETD2 weights have no adjoint.
"""
from __future__ import annotations

import math

import torch

from . import _native as nat
from . import autotune

__all__ = ["RK4Rollout", "RK3Rollout", "ETD2Rollout", "shell_spectrum", "log_spectrum_misfit"]

_SIZES = (16, 24, 32, 48, 64, 96, 128, 256, 512)


class RK4Rollout:
    METHOD = "RK4"

    def __init__(self, n, nu, dt, les="Smagorinsky", Cs=0.17, dtype=torch.float32, parity=True, forcing=0.0,
                 checkpoint_every=10, device="cuda"):
        if int(n) not in _SIZES:
            raise ValueError("grid N=%d is not compiled (supported: %s)" % (n, _SIZES))
        if checkpoint_every < 1:
            raise ValueError("checkpoint_every must be >= 1")
        self.n, self.nu, self.dt = int(n), float(nu), float(dt)
        self.forcing, self.every = float(forcing), int(checkpoint_every)
        model = nat.LES_NONE
        if les is not None:
            if les[0] not in "SsVv":
                raise ValueError("LES model must be 'Smagorinsky' or 'vreman'")
            model = nat.LES_SMAGORINSKY if les[0] in "Ss" else nat.LES_VREMAN
        self.les = model
        self.Cs = float(Cs)
        self.rdtype = dtype
        self.cdtype = torch.complex64 if dtype == torch.float32 else torch.complex128
        self.device = torch.device(device)
        scheme = nat.SCHEME_RK4 if self.METHOD == "RK4" else nat.SCHEME_RK3
        self.ns = 4 if self.METHOD == "RK4" else 3  # stages per step
        self.plan = nat.Plan(3, self.n, dtype, model, scheme, parity, nu, Cs, forcing, self.device)
        autotune.apply_cached(self.plan, self.METHOD)
        self.nk, self.nkp = self.plan.nk, self.plan.nkp
        self._ws_owner, self._ws = self.plan.adjoint_workspace()
        self._store = []   # stage states of the segment being reversed (reused across calls)

    # ---- storage helpers ----
    def _new(self):
        return torch.zeros((3, self.n, self.n, self.nkp), dtype=self.cdtype, device=self.device)

    def _pad(self, U):
        s = self._new()
        s[..., : self.nk].copy_(U.detach().to(self.cdtype))
        return s

    def rfft(self, u):
        """(3, n, n, n) real -> (3, n, n, n//2+1) complex with this rollout's own r2c."""
        u = torch.as_tensor(u, device=self.device).to(self.rdtype).contiguous()
        s = self._new()
        self.plan.fft_r2c(u, s, 3)
        return s[..., : self.nk].clone()

    # ---- forward ----
    def _flags(self, rk, primed):
        f = nat.STAGE_PRIMED if (primed and rk == 0) or rk > 0 else 0
        return f | (nat.STAGE_RK4 if self.ns == 4 else 0)

    def _step(self, A, B, Cacc, primed):
        """One fused step from A (kept) into B; Cacc is the RK4 accumulator
        (overwritten).  Returns True (the workspace is primed with B)."""
        if self.ns == 4:
            Cacc.copy_(A)  # U_hat1 = U_hat at step entry (SM_solver.py:33)
        for rk in range(self.ns):
            self.plan.stage(rk, self.dt, A if rk == 0 else B, A, Cacc if self.ns == 4 else None, B, None, None,
                            None, self._flags(rk, primed))
        return True

    def _step_keep(self, A, stages, Cacc, primed):
        """As _step, writing the stage states U_1..U_{ns-1} to stages[0..ns-2]
        and the step output to stages[ns-1]."""
        if self.ns == 4:
            Cacc.copy_(A)
        cur = A
        for rk in range(self.ns):
            self.plan.stage(rk, self.dt, cur, A, Cacc if self.ns == 4 else None, stages[rk], None, None, None,
                            self._flags(rk, primed))
            cur = stages[rk]
        return True

    def forward_states(self, U0, Cs, nsteps):
        """Run ``nsteps`` fused RK4 steps; return (U_T padded, checkpoints)."""
        self.plan.set_params(self.nu, Cs, self.forcing)
        A, B, Cacc = self._pad(U0), self._new(), self._new()
        ckpts = {0: A.clone()}
        primed = False
        for k in range(int(nsteps)):
            primed = self._step(A, B, Cacc, primed)
            A, B = B, A
            if (k + 1) % self.every == 0 and (k + 1) < nsteps:
                ckpts[k + 1] = A.clone()
        return A, ckpts

    # ---- backward ----
    def backward_states(self, ckpts, gUT, Cs, nsteps):
        """Reverse sweep; returns (dL/dU_0 padded, dL/dCs float64 tensor)."""
        self.plan.set_params(self.nu, Cs, self.forcing)
        dt = self.dt
        ubar, acc, lam = self._pad(gUT), self._new(), self._new()
        csg = torch.zeros(1, dtype=torch.float64, device=self.device)
        self.plan.adjoint_seed(self._ws, dt, ubar, acc, lam)
        starts = sorted(ckpts)
        ends = starts[1:] + [int(nsteps)]
        Cacc = self._new()
        store = self._store
        while len(store) < max(e - s for s, e in zip(starts, ends)):
            store.append([self._new() for _ in range(self.ns)])
        last = self.ns - 1
        for s0, s1 in reversed(list(zip(starts, ends))):
            m = s1 - s0
            # recompute the segment: inputs[i] = state entering step s0 + i
            inputs = [ckpts[s0]]
            primed = False
            for i in range(m):
                primed = self._step_keep(inputs[i], store[i], Cacc, primed)
                inputs.append(store[i][last])
            # stage states of step i: U_0 = inputs[i], U_1..U_last = store[i][0..last-1]
            states = lambda i, s: inputs[i] if s == 0 else store[i][s - 1]
            self.plan.adjoint_prime(self._ws, states(m - 1, last), lam)
            for i in range(m - 1, -1, -1):
                for s in range(last, -1, -1):
                    if s > 0:
                        un = states(i, s - 1)
                    else:
                        un = states(i - 1, last) if i > 0 else None
                    self.plan.adjoint_stage(self._ws, s, dt, un, ubar, acc, lam, csg)
        # a bounded wait that gave up (forward recompute or reverse passes) raises here
        self.plan.check()
        self.plan.adjoint_check(self._ws)
        return ubar, csg

    def __call__(self, U0, Cs, nsteps):
        if not torch.is_tensor(Cs):
            Cs = torch.tensor(float(Cs), dtype=torch.float64, device=self.device)
        return _RolloutFn.apply(U0, Cs, self, int(nsteps))

    def timed(self, U0, Cs, nsteps, gUT):
        """(forward ms, backward ms, U_T, dL/dU_0, dL/dCs) of one rollout and its
        reverse sweep, timed with CUDA events on the current stream."""
        st = torch.cuda.current_stream(self.device)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize(self.device)
        e[0].record(st)
        UT, ck = self.forward_states(U0, float(Cs), nsteps)
        e[1].record(st)
        g, c = self.backward_states(ck, gUT, float(Cs), nsteps)
        e[2].record(st)
        torch.cuda.synchronize(self.device)
        return e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2]), UT, g, c


class RK3Rollout(RK4Rollout):
    """The reference's RK3 (src/RK3_method.py:20-41, ``parity=True``) or the
    corrected SSP-RK3 (``parity=False``) with its discrete adjoint; same
    arguments and use as ``RK4Rollout``."""
    METHOD = "RK3"


class ETD2Rollout:
    """Corrected ETD2 with its discrete adjoint (3D).  The first step records
    F(U_0) and runs RK4 (src/ETD2_method.py:7-14); later steps are
    U_{n+1} = E U_n + w1 F(U_n) + w0 F(U_{n-1}) with E = exp(-dt nu k^2) and
    F the explicit term (projected u x omega, LES stress, forcing).  The
    forward keeps (U_n, F(U_{n-1})) every ``checkpoint_every`` steps; the
    backward recomputes one segment at a time and runs the ETD2 reverse steps
    on this plan and the first step's RK4 reverse on a companion RK4 plan.
    Same call and gradient conventions as ``RK4Rollout``.
    """

    def __init__(self, n, nu, dt, les="Smagorinsky", Cs=0.17, dtype=torch.float32, forcing=0.0,
                 checkpoint_every=10, device="cuda"):
        if checkpoint_every < 1:
            raise ValueError("checkpoint_every must be >= 1")
        self.rk = RK4Rollout(n, nu, dt, les=les, Cs=Cs, dtype=dtype, forcing=forcing, checkpoint_every=1,
                             device=device)
        self.n, self.nu, self.dt, self.forcing = self.rk.n, self.rk.nu, self.rk.dt, self.rk.forcing
        self.every = int(checkpoint_every)
        self.rdtype, self.cdtype, self.device = self.rk.rdtype, self.rk.cdtype, self.rk.device
        self.plan = nat.Plan(3, self.n, dtype, self.rk.les, nat.SCHEME_ETD2, False, nu, Cs, forcing, self.device)
        autotune.apply_cached(self.plan, "ETD2")
        self.nk, self.nkp = self.plan.nk, self.plan.nkp
        self._ws_owner, self._ws = self.plan.adjoint_workspace()
        self.rfft = self.rk.rfft

    def _new(self):
        return self.rk._new()

    def _steps(self, U_start, F_prev, k0, k1, keep=None, ckpts=None):
        """Steps k0 .. k1-1 from U_{k0} (F_prev = F(U_{k0-1}) when k0 >= 1);
        appends each step's input state to ``keep`` and records checkpoints
        (U_k, F(U_{k-1})) in ``ckpts``.  Returns U_{k1}."""
        U = U_start.clone()
        if k0 == 0:
            F1, tmp = self._new(), self._new()
            self.plan.rhs(U, tmp, F1)  # F(U_0), src/ETD2_method.py:8-14
            if keep is not None:
                keep.append(U.clone())
            if ckpts is not None:
                ckpts[0] = (U.clone(), None)
            B, Cacc = self._new(), self._new()
            self.rk._step(U, B, Cacc, False)  # first step: RK4
            U, F0, k = B, tmp, 1
        else:
            F1, F0, k = F_prev.clone(), self._new(), k0
        primed = False
        while k < k1:
            if keep is not None:
                keep.append(U.clone())
            if ckpts is not None and k % self.every == 0:
                ckpts[k] = (U.clone(), F1.clone())
            # U <- E U + w1 F(U) + w0 F1; F0 <- F(U) (src/ETD2_method.py:16-37)
            self.plan.stage(0, self.dt, U, None, F1, U, F0, None, None, nat.STAGE_PRIMED if primed else 0)
            primed = True
            F0, F1 = F1, F0
            k += 1
        return U

    def forward_states(self, U0, Cs, nsteps):
        """Run ``nsteps`` steps; return (U_T padded, checkpoints)."""
        nsteps = int(nsteps)
        if nsteps < 1:
            raise ValueError("nsteps must be >= 1")
        for p in (self.plan, self.rk.plan):
            p.set_params(self.nu, Cs, self.forcing)
        ckpts = {}
        U = self._steps(self.rk._pad(U0), None, 0, nsteps, ckpts=ckpts)
        return U, ckpts

    def backward_states(self, ckpts, gUT, Cs, nsteps):
        """Reverse sweep; returns (dL/dU_0 padded, dL/dCs float64 tensor)."""
        nsteps = int(nsteps)
        for p in (self.plan, self.rk.plan):
            p.set_params(self.nu, Cs, self.forcing)
        csg = torch.zeros(1, dtype=torch.float64, device=self.device)
        ubar = self.rk._pad(gUT)
        lam, acc = self._new(), self._new()
        if nsteps > 1:
            self.plan.adjoint_seed(self._ws, self.dt, ubar, acc, lam)  # lam = w1 ubar
            starts = sorted(ckpts)
            ends = starts[1:] + [nsteps]
            for s0, s1 in reversed(list(zip(starts, ends))):
                states = []  # U_{s0} .. U_{s1-1}
                U_s, F_prev = ckpts[s0]
                self._steps(U_s, F_prev, s0, s1, keep=states)
                lo = max(s0, 1)
                for k in range(s1 - 1, lo - 1, -1):
                    if k == s1 - 1:
                        self.plan.adjoint_prime(self._ws, states[k - s0], lam)
                    un = states[k - 1 - s0] if k - 1 >= lo else None
                    # stage 0: a reverse ETD2 step; 1: the step after the RK4 step, which
                    # leaves lam = the cotangent of F(U_0)
                    self.plan.adjoint_stage(self._ws, 0 if k > 1 else 1, self.dt, un, ubar, acc, lam, csg)
        # the RK4 step's reverse from dL/dU_1
        g, c = self.rk.backward_states({0: ckpts[0][0]}, ubar[..., : self.nk], Cs, 1)
        if nsteps > 1:  # + J_F(U_0)^T (cotangent of F(U_0))
            self.plan.adjoint_prime(self._ws, ckpts[0][0], lam)
            self.plan.adjoint_stage(self._ws, 2, self.dt, None, g, acc, lam, csg)
        self.plan.check()
        self.plan.adjoint_check(self._ws)
        return g, csg + c

    def __call__(self, U0, Cs, nsteps):
        if not torch.is_tensor(Cs):
            Cs = torch.tensor(float(Cs), dtype=torch.float64, device=self.device)
        return _RolloutFn.apply(U0, Cs, self, int(nsteps))


class _RolloutFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U0, Cs, ro, nsteps):
        UT, ckpts = ro.forward_states(U0, float(Cs), nsteps)
        ctx.ro, ctx.ckpts, ctx.nsteps, ctx.cs = ro, ckpts, nsteps, float(Cs)
        ctx.u_dtype, ctx.cs_dtype = U0.dtype, Cs.dtype
        return UT[..., : ro.nk].clone()

    @staticmethod
    def backward(ctx, gUT):
        ro = ctx.ro
        g, csg = ro.backward_states(ctx.ckpts, gUT.contiguous(), ctx.cs, ctx.nsteps)
        ctx.ckpts = None
        gU = g[..., : ro.nk].clone().to(ctx.u_dtype)
        return gU, csg[0].to(ctx.cs_dtype), None, None


def shell_spectrum(U_hat, n, nshells=None):
    """E(k) on integer shells round(|k|): 1/2 sum w |u_hat|^2 / N^6, w = 2 on
    0 < kz < N/2, in float64 (differentiable torch ops)."""
    dev = U_hat.device
    kc = (torch.fft.fftfreq(n, device=dev, dtype=torch.float64) * n).round()
    kz = torch.arange(n // 2 + 1, device=dev, dtype=torch.float64)
    K2 = kc.view(n, 1, 1) ** 2 + kc.view(1, n, 1) ** 2 + kz.view(1, 1, -1) ** 2
    w = torch.where((kz > 0) & (kz < n // 2), 2.0, 1.0).view(1, 1, -1)
    rd = torch.float64  # accumulated in float64 whatever the state's precision
    ur, ui = U_hat.real.to(rd), U_hat.imag.to(rd)
    e = 0.5 * w * (ur * ur + ui * ui).sum(0) / float(n) ** 6
    shell = torch.round(torch.sqrt(K2)).long().reshape(-1)
    ns = int(shell.max()) + 1 if nshells is None else int(nshells)
    keep = shell < ns
    return torch.zeros(ns, dtype=rd, device=dev).index_add(0, shell[keep], e.reshape(-1)[keep])


def log_spectrum_misfit(U_hat, E_target, n, kmin=1, kmax=None):
    """sum_{k=kmin..kmax} (log E(k) - log E_target(k))^2, kmax = floor(2/3 (N/2+1))."""
    kmax = int(math.floor(2.0 / 3.0 * (n // 2 + 1))) if kmax is None else int(kmax)
    E = shell_spectrum(U_hat, n, kmax + 1)
    Et = torch.as_tensor(E_target, device=U_hat.device)[: kmax + 1].to(E.dtype)
    d = torch.log(E[kmin: kmax + 1]) - torch.log(Et[kmin: kmax + 1])
    return (d * d).sum()
