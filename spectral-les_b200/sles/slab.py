"""One 3D domain decomposed in slabs over P ranks, one GPU each.

The reference distributes its fields with mpi4py-fft's PFFT in slabs
(src/initialize_domain.py:59-65, bounds src/utilites.py:18-24): physical
space split along x, spectral space along y, with a global transpose (an
all-to-all) inside every 3D transform, and u_max all-reduced for the CFL
step (src/SM_solver.py:245-255).  Here rank r holds the ky rows
[r m, (r+1) m) of every spectral field (m = N/P) and one RHS evaluation is

  x inverse of the state on the ky rows        sles_slab_prime, or the
                                                previous stage's x pass
  exchange 1: ky rows -> x planes              all-to-all per field
  y inverse, fused z pass, y forward           sles_slab_middle
  exchange 2: x planes -> ky rows              all-to-all per field
  x forward, projection, stage update,         sles_slab_stage
  x inverse of the new state

The exchanges are ``torch.distributed.all_to_all_single`` on the current
stream (NCCL over NVLink on GPUs); ``exchange`` may be replaced (tests run
the P ranks of one domain inside one process with copies between their
buffers).  Schemes: the reference's RK3, SSP-RK3 and RK4, with or without
LES, float32 or float64.

    sd = SlabDomain(256, nu=1e-4, dt=1e-3, method="RK3", les="Smagorinsky", Cs=0.17,
                    nranks=dist.get_world_size(), rank=dist.get_rank())
    sd.set_state(U_hat_full)      # (3, N, N, N//2+1) complex: this rank keeps its ky rows
    sd.step()
    U = sd.gather()               # the whole field on every rank
"""
from __future__ import annotations

import struct

import torch

from . import _native as nat

__all__ = ["SlabDomain", "emulated_exchange", "umax_decode"]


def umax_decode(bits):
    """The z pass's ordered 64-bit encoding of a double back to the value."""
    b = int(bits) & 0xFFFFFFFFFFFFFFFF
    if b == 0:
        return float("-inf")
    u = (b & 0x7FFFFFFFFFFFFFFF) if (b >> 63) else (~b & 0xFFFFFFFFFFFFFFFF)
    return struct.unpack("<d", struct.pack("<Q", u))[0]


def _nccl_exchange(group):
    import torch.distributed as dist

    def ex(out, inp):
        dist.all_to_all_single(out, inp, group=group)
    return ex


class SlabDomain:
    def __init__(self, n, nu=0.01, dt=0.01, method="RK3", les=None, Cs=0.17, dtype=torch.float32, parity=True,
                 nranks=1, rank=0, device="cuda", exchange=None, group=None, plan_factory=None):
        if method not in ("RK3", "RK4"):
            raise ValueError("slab domains step RK3 or RK4")
        self.N, self.P, self.r = int(n), int(nranks), int(rank)
        self.nu, self.dt, self.method, self.Cs = float(nu), float(dt), method, float(Cs)
        self.device = torch.device(device)
        self.rdtype = dtype
        self.cdtype = torch.complex64 if dtype == torch.float32 else torch.complex128
        model = nat.LES_NONE
        if les is not None:
            model = nat.LES_SMAGORINSKY if les[0] in "Ss" else nat.LES_VREMAN
        scheme = nat.SCHEME_RK3 if method == "RK3" else nat.SCHEME_RK4
        # plan_factory: a stand-in with the same slab entry points (tests on CPU)
        make = plan_factory if plan_factory is not None else nat.Plan
        self.plan = make(3, self.N, dtype, model, scheme, parity, nu, Cs, 0.0, self.device, slab=(self.P, self.r))
        info = self.plan.slab_info()
        self.m, self.n1, self.n2 = info.m, info.n_exchange1, info.n_exchange2
        self.block, self.field = int(info.block_elems), int(info.field_elems)
        self.nk, self.nkp = self.plan.nk, self.plan.nkp
        ws = self.plan.workspace
        esz = torch.empty((), dtype=self.cdtype).element_size()

        def view(addr, nf):  # nf fields of P blocks inside the workspace
            off = addr - ws.data_ptr()
            return ws[off: off + nf * self.field * esz].view(self.cdtype).view(nf, self.P * self.block)
        s1, r1, s2, r2 = self.plan.slab_buffers()
        self.send1, self.recv1 = view(s1, self.n1), view(r1, self.n1)
        self.send2, self.recv2 = view(s2, self.n2), view(r2, self.n2)
        self.exchange = exchange if exchange is not None else _nccl_exchange(group)
        self.group = group
        shape = (3, self.N, self.m, self.nkp)
        self.U_hat = torch.zeros(shape, dtype=self.cdtype, device=self.device)
        self._u0 = torch.zeros_like(self.U_hat)
        self._u1 = torch.zeros_like(self.U_hat) if method == "RK4" else None
        self._umax = torch.zeros(1, dtype=torch.int64, device=self.device)
        self._primed = None
        self.u_max = None  # max over ranks of u at the start of the last step (after step())

    # ---- state ----
    def set_state(self, U_hat_full):
        """This rank's ky rows of a whole half-complex field (3, N, N, >= N//2+1)."""
        src = torch.as_tensor(U_hat_full, device=self.device)
        rows = slice(self.r * self.m, (self.r + 1) * self.m)
        self.U_hat.zero_()
        self.U_hat[..., : self.nk].copy_(src[:, :, rows, : self.nk].to(self.cdtype))
        if self._u1 is not None:
            self._u1.copy_(self.U_hat)
        self._primed = None

    def local(self):
        """This rank's slab of U_hat: (3, N, m, N//2+1)."""
        return self.U_hat[..., : self.nk]

    def gather(self):
        """The whole U_hat (3, N, N, N//2+1) on every rank (torch.distributed all_gather)."""
        if self.P == 1:
            return self.local().clone()
        import torch.distributed as dist
        parts = [torch.empty_like(self.U_hat) for _ in range(self.P)]
        dist.all_gather(parts, self.U_hat.contiguous(), group=self.group)
        return torch.cat(parts, dim=2)[..., : self.nk]

    # ---- one RHS evaluation + stage update ----
    def _ex1(self):
        for f in range(self.n1):
            self.exchange(self.recv1[f], self.send1[f])

    def _ex2(self):
        for f in range(self.n2):
            self.exchange(self.recv2[f], self.send2[f])

    def _stage(self, k, ucur, u0, u1, uout, flags, umax=None):
        if self._primed != (ucur.data_ptr(), ucur._version):
            self.plan.slab_prime(ucur)
        self._ex1()
        self.plan.slab_middle(umax)
        self._ex2()
        self.plan.slab_stage(k, self.dt, ucur, u0, u1, uout, None, flags)
        self._primed = (uout.data_ptr(), uout._version)

    def step(self):
        """One step of the scheme (src/RK3_method.py:20-41 / SSP-RK3, or
        src/RK4_method.py:20-35 with U_hat1 = U_hat kept by the domain)."""
        A, B = self.U_hat, self._u0
        self._umax.zero_()
        if self.method == "RK3":
            for rk in range(3):
                self._stage(rk, A if rk == 0 else B, A, None, B, 0, self._umax if rk == 0 else None)
        else:
            C = self._u1
            for rk in range(4):
                self._stage(rk, A if rk == 0 else B, A, C, B, nat.STAGE_RK4, self._umax if rk == 0 else None)
        self.U_hat, self._u0 = B, A
        self._primed = (B.data_ptr(), B._version)
        self.u_max = self._reduce_umax()

    def _reduce_umax(self):
        v = torch.tensor([umax_decode(self._umax.item())], dtype=torch.float64, device=self.device)
        if self.P > 1:
            import torch.distributed as dist
            if dist.is_initialized():
                dist.all_reduce(v, op=dist.ReduceOp.MAX, group=self.group)  # src/SM_solver.py:254
        return float(v.item())

    def check(self):
        return self.plan.check()


def emulated_exchange(domains):
    """Exchanges for P SlabDomains of one decomposition living in one process
    (one GPU): the all-to-all done by copies between their buffers.  Returns
    a stepping function advancing all of them by one step in lockstep."""
    P = len(domains)

    def run_stage(d_stage_args):
        for d, (k, ucur, u0, u1, uout, flags, umax) in zip(domains, d_stage_args):
            if d._primed != (ucur.data_ptr(), ucur._version):
                d.plan.slab_prime(ucur)
        _copy(lambda d: d.send1, lambda d: d.recv1, "n1")
        for d, a in zip(domains, d_stage_args):
            d.plan.slab_middle(a[6])
        _copy(lambda d: d.send2, lambda d: d.recv2, "n2")
        for d, (k, ucur, u0, u1, uout, flags, umax) in zip(domains, d_stage_args):
            d.plan.slab_stage(k, d.dt, ucur, u0, u1, uout, None, flags)
            d._primed = (uout.data_ptr(), uout._version)

    def _copy(src, dst, nattr):
        for q in range(P):  # rank q receives block r of every field from rank r
            for r in range(P):
                b = domains[0].block
                for f in range(getattr(domains[0], nattr)):
                    dst(domains[q])[f, r * b:(r + 1) * b].copy_(src(domains[r])[f, q * b:(q + 1) * b])

    def step():
        nst = 3 if domains[0].method == "RK3" else 4
        bufs = [(d.U_hat, d._u0, d._u1) for d in domains]
        for d in domains:
            d._umax.zero_()
        for rk in range(nst):
            args = []
            for d, (A, B, C) in zip(domains, bufs):
                flags = nat.STAGE_RK4 if d.method == "RK4" else 0
                args.append((rk, A if rk == 0 else B, A, C, B, flags, d._umax if rk == 0 else None))
            run_stage(args)
        for d, (A, B, C) in zip(domains, bufs):
            d.U_hat, d._u0 = B, A
            d._primed = (B.data_ptr(), B._version)
        vals = [umax_decode(d._umax.item()) for d in domains]
        for d in domains:
            d.u_max = max(vals)
    return step
