"""The plain GPU path: the reference's right-hand side and integrators written
with torch.fft (cuFFT on a GPU) and unfused torch elementwise ops.

This is the comparison path the fused kernels are measured against (the
"plain FP64 GPU path") and, being ordinary differentiable torch code, the
autograd reference for the hand-written adjoint.  It is not used by the
drop-in API.

Conventions follow the reference (src/initialize_domain.py:76-114, 162-167):
kx = fftfreq(N)*N on the full axes, the r2c (last) axis keeps its Nyquist bin
at +N/2, mask = prod_i [|k_i| < 2/3 (N/2+1)], K_over_K2 with K2 = 0 -> 1.

    ps = PlainSolver(n=64, nu=1e-4, dt=1e-3, les="Smagorinsky", Cs=0.17, method="RK4")
    Uh = ps.rfft(u)                  # (3, n, n, n//2+1) complex
    Uh = ps.step(Uh)                 # one reference RK4 step
"""
from __future__ import annotations

import math

import torch
from torch.utils.checkpoint import checkpoint

__all__ = ["PlainSolver"]


class PlainSolver:
    def __init__(self, n, dim=3, nu=0.0, dt=0.01, les=None, Cs=0.17, method="RK4", parity=True,
                 forcing=0.0, dtype=torch.float64, device=None):
        if method not in ("RK4", "RK3", "ETD2"):
            raise ValueError("Invalid method name")
        if les is not None and les[0] not in "SsVv":
            raise ValueError("LES model must be 'Smagorinsky' or 'vreman'")
        if method == "ETD2" and parity:
            raise ValueError("the plain path implements the corrected ETD2 only (parity=False)")
        self.n, self.dim, self.nu, self.dt = int(n), int(dim), float(nu), float(dt)
        self.les = None if les is None else ("S" if les[0] in "Ss" else "V")
        self.Cs, self.method, self.parity, self.forcing = float(Cs), method, bool(parity), float(forcing)
        self.rdtype = dtype
        self.device = torch.device(device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu"))
        self.dx = 2.0 * math.pi / self.n
        n, dev = self.n, self.device
        kc = (torch.fft.fftfreq(n, device=dev, dtype=torch.float64) * n).round()
        kr = torch.arange(n // 2 + 1, device=dev, dtype=torch.float64)   # last axis: Nyquist at +N/2
        shp = [1] * dim
        self.K = []
        for i in range(dim):
            s = list(shp)
            s[i] = -1
            self.K.append((kc if i < dim - 1 else kr).reshape(s).to(dtype))
        K2 = sum(k * k for k in self.K)
        self.K2 = K2
        K2d = torch.where(K2 == 0, torch.ones_like(K2), K2)
        self.KoK2 = [k / K2d for k in self.K]
        kmax = 2.0 / 3.0 * (n // 2 + 1)
        m = torch.ones_like(K2, dtype=torch.bool)
        for k in self.K:
            m = m & (k.abs() < kmax)
        self.mask = m.to(dtype)
        self.nonzero = (K2 != 0).to(dtype)
        self.first = True
        if method == "ETD2":
            z = dt * nu * K2.to(torch.float64)
            E = torch.exp(-z)
            zz = torch.where(z == 0, torch.ones_like(z), z)
            c1 = dt * ((1.0 - zz) * torch.exp(-zz) - 1.0 + 2.0 * zz) / (zz * zz)
            c0 = dt * (-torch.exp(-zz) + 1.0 - zz) / (zz * zz)
            small = z.abs() < 1e-2
            c1 = torch.where(small, dt * (1.5 - 2.0 * z / 3.0 + z * z / 4.0 - z ** 3 / 15.0), c1)
            c0 = torch.where(small, dt * (-0.5 + z / 6.0 - z * z / 24.0 + z ** 3 / 120.0), c0)
            self.E, self.c1, self.c0 = (x.to(dtype) for x in (E, c1, c0))

    # ---- transforms ----
    def rfft(self, a):
        return torch.fft.rfftn(a, dim=tuple(range(-self.dim, 0)))

    def irfft(self, a):
        return torch.fft.irfftn(a, s=(self.n,) * self.dim, dim=tuple(range(-self.dim, 0)))

    # ---- operators (src/math_formula.py) ----
    def gradient(self, Uh):
        """A[i][j] = d u_j / d x_i (math_formula.py:27-62)."""
        return [[self.irfft(1j * self.K[i] * Uh[j]) for j in range(self.dim)] for i in range(self.dim)]

    def curl(self, Uh):
        """math_formula.py:16-25."""
        K = self.K
        if self.dim == 2:
            return self.irfft(1j * (K[0] * Uh[1] - K[1] * Uh[0]))
        return torch.stack([self.irfft(1j * (K[1] * Uh[2] - K[2] * Uh[1])),
                            self.irfft(1j * (K[2] * Uh[0] - K[0] * Uh[2])),
                            self.irfft(1j * (K[0] * Uh[1] - K[1] * Uh[0]))])

    def u_cross_omega(self, U, w):
        """math_formula.py:5-13."""
        if self.dim == 2:
            return torch.stack([self.rfft(U[1] * w), self.rfft(-U[0] * w)])
        return torch.stack([self.rfft(U[1] * w[2] - U[2] * w[1]), self.rfft(U[2] * w[0] - U[0] * w[2]),
                            self.rfft(U[0] * w[1] - U[1] * w[0])])

    def eddy_viscosity(self, A, Cs):
        """smagorinsky.py:24-47, vreman.py:30-147 (thresholds kept, B not clamped)."""
        d = self.dim
        if self.les == "S":
            ss = 0
            for i in range(d):
                ss = ss + A[i][i] * A[i][i]
                for j in range(i + 1, d):
                    ss = ss + 0.5 * (A[i][j] + A[j][i]) ** 2
            return torch.sqrt(2.0 * ss) * (Cs * self.dx) ** 2
        b = [[sum(A[m][p] * A[m][q] for m in range(d)) for q in range(d)] for p in range(d)]
        if d == 3:
            B = (b[0][0] * b[1][1] - b[0][1] * b[0][1] + b[0][0] * b[2][2] - b[0][2] * b[0][2]
                 + b[1][1] * b[2][2] - b[1][2] * b[1][2])
        else:
            B = b[0][0] * b[1][1] - b[0][1] * b[0][1]
        sb = torch.sqrt(B)
        aa = sum(A[i][j] * A[i][j] for i in range(d) for j in range(d))
        gate = (aa > 10e-5) & (sb > aa / 10e6)
        return sb * torch.where(gate, torch.sqrt(1.0 / aa), torch.zeros_like(aa)) * (2.5 * Cs * Cs * self.dx * self.dx)

    def stress(self, Uh, Cs):
        """T_i = 2i mask sum_j K_j rfftn(nu_t S_ij) (math_formula.py:64-127); in 2D the
        corrected form (both components)."""
        A = self.gradient(Uh)
        nu = self.eddy_viscosity(A, Cs)
        d = self.dim
        S = lambda i, j: A[i][i] if i == j else 0.5 * (A[i][j] + A[j][i])
        F = {}
        for i in range(d):
            for j in range(i, d):
                F[(i, j)] = F[(j, i)] = self.rfft(S(i, j) * nu)
        return torch.stack([sum(self.K[j] * F[(i, j)] for j in range(d)) * (2j * self.mask) for i in range(d)])

    def projected_nonlinear(self, Uh, Cs=None):
        """P(mask N_hat [+ T_hat])."""
        Cs = self.Cs if Cs is None else Cs
        N = self.u_cross_omega(self.irfft(Uh), self.curl(Uh)) * self.mask
        if self.les:
            N = N + self.stress(Uh, Cs)
        P = sum(N[i] * self.KoK2[i] for i in range(self.dim))
        return torch.stack([N[i] - P * self.K[i] for i in range(self.dim)])

    def rhs(self, Uh, Cs=None):
        """computeRHS, src/RK4_method.py:38-71."""
        Cs = self.Cs if Cs is None else Cs
        dU = self.u_cross_omega(self.irfft(Uh), self.curl(Uh)) * self.mask
        T = self.stress(Uh, Cs) if self.les else None
        R = dU + T if self.les else dU
        P = sum(R[i] * self.KoK2[i] for i in range(self.dim))
        dU = torch.stack([dU[i] - P * self.K[i] for i in range(self.dim)])
        if self.forcing > 0.0:
            dU = dU + self.forcing * Uh * self.nonzero
        if self.nu > 0.0:
            dU = dU - self.nu * self.K2 * Uh
        if self.les:
            dU = dU + T
        return dU

    # ---- integrators ----
    def rk4(self, Uh, Cs=None):
        """src/RK4_method.py:20-35 (U_hat1 = U_hat on entry)."""
        dt = self.dt
        U0, U1, U = Uh, Uh, Uh
        a, b = [1 / 6, 1 / 3, 1 / 3, 1 / 6], [0.5, 0.5, 1.0]
        for rk in range(4):
            dU = self.rhs(U, Cs)
            if rk < 3:
                U = U0 + b[rk] * dt * dU
            U1 = U1 + a[rk] * dt * dU
        return U1

    def rk3(self, Uh, Cs=None):
        """src/RK3_method.py:20-41 (parity) or SSP-RK3 (Shu & Osher 1988)."""
        dt, U0 = self.dt, Uh
        if self.parity:
            dU = self.rhs(U0, Cs)
            U = U0 + 0.5 * dt * dU
            dU = self.rhs(U, Cs)
            U = U0 - dt * dU + 2.0 * dt * dU
            dU = self.rhs(U, Cs)
            return U0 + dt * (1 / 6 * dU + 2 / 3 * dU + 1 / 6 * dU)
        U = U0 + dt * self.rhs(U0, Cs)
        U = 0.75 * U0 + 0.25 * (U + dt * self.rhs(U, Cs))
        return (1.0 / 3.0) * U0 + (2.0 / 3.0) * (U + dt * self.rhs(U, Cs))

    def step(self, Uh, Cs=None):
        """One step of ``method``.  ETD2 (corrected, Cox & Matthews 2002): the
        first step records F1 and runs RK4 (src/ETD2_method.py:7-14); later
        steps use the exponential integrator with the stored F1."""
        if self.method == "RK4":
            return self.rk4(Uh, Cs)
        if self.method == "RK3":
            return self.rk3(Uh, Cs)
        if self.first:
            self.F1 = self.projected_nonlinear(Uh, Cs)
            self.first = False
            return self.rk4(Uh, Cs)
        F0, self.F1 = self.F1, self.projected_nonlinear(Uh, Cs)
        return Uh * self.E + self.F1 * self.c1 + F0 * self.c0

    def rollout(self, Uh, nsteps, Cs=None, checkpoint_steps=False):
        """``nsteps`` RK steps (RK3/RK4).  checkpoint_steps: keep only each step's
        input for autograd and recompute the step's interior on backward."""
        if self.method == "ETD2":
            raise ValueError("rollout: RK3/RK4 only")
        f = self.rk4 if self.method == "RK4" else self.rk3
        for _ in range(int(nsteps)):
            Uh = checkpoint(f, Uh, Cs, use_reentrant=False) if checkpoint_steps else f(Uh, Cs)
        return Uh

    # ---- diagnostics ----
    def hermitian_weights(self):
        kz = self.K[-1]
        return torch.where((kz != 0) & (kz != self.n // 2), 2.0, 1.0).to(self.rdtype)

    def shell_spectrum(self, Uh, nshells=None):
        """E(k) on integer shells round(|k|): 1/2 sum w |u_hat|^2 / N^(2d) (differentiable)."""
        e = 0.5 * self.hermitian_weights() * (Uh.real ** 2 + Uh.imag ** 2).sum(0) / float(self.n) ** (2 * self.dim)
        shell = torch.round(torch.sqrt(self.K2.to(torch.float64))).long().expand_as(e).reshape(-1)
        ns = int(shell.max()) + 1 if nshells is None else int(nshells)
        keep = shell < ns
        out = torch.zeros(ns, dtype=e.dtype, device=e.device)
        return out.index_add(0, shell[keep], e.reshape(-1)[keep])
