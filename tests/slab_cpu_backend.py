"""A CPU stand-in for the slab entry points of libsles_b200 (test helper).

Implements, with torch.fft on CPU tensors, the contract include/sles.h gives
sles_slab_prime / sles_slab_middle / sles_slab_stage for a slab plan -- which
fields go where, in which layout, unscaled transforms with the 1/N^3 on the
c2r -- so that the decomposition logic of sles.slab.SlabDomain (the
exchange blocks, the ky-row offsets, the stage sequencing, the u_max
reduction) can run over gloo ranks without a GPU.  Reference RK3 with the
Smagorinsky closure (src/RK3_method.py:20-77, src/smagorinsky.py:24-47,
src/math_formula.py:5-127); the GPU kernels are checked separately.
"""
import math

import torch

from sles import _native as nat


class CpuSlabPlan:
    def __init__(self, dim, n, dtype, les_model, scheme, parity, nu, cs, forcing, device, slab=None):
        assert dim == 3 and les_model == nat.LES_SMAGORINSKY and scheme == nat.SCHEME_RK3 and parity
        self.N, (self.P, self.r) = n, slab
        self.m = n // self.P
        self.nu, self.cs = nu, cs
        self.nk = n // 2 + 1
        self.nkp = (self.nk + 3) // 4 * 4
        self.cdtype = torch.complex128
        self.device = torch.device("cpu")
        self.field = n * self.m * self.nkp
        self.block = self.m * self.m * self.nkp
        self.n1 = self.n2 = 6
        nslots = 9 + self.n1 + self.n2
        self.workspace = torch.zeros(nslots * self.field * 16, dtype=torch.uint8)
        self._c = self.workspace.view(torch.complex128).view(nslots, self.field)
        kc = (torch.fft.fftfreq(n, dtype=torch.float64) * n).round()
        self.kc = kc
        self.kz = torch.arange(self.nk, dtype=torch.float64)
        self.kmax = 2.0 / 3.0 * (n // 2 + 1)
        self._umax_store = None

    # ---- contract of include/sles.h ----
    def slab_info(self):
        return nat.SlabLayout(self.P, self.r, self.m, self.n1, self.n2, 0, self.block, self.field)

    def slab_buffers(self):
        b = self._c.data_ptr()
        fb = self.field * 16
        return [b, b + 9 * fb, b + (9 + self.n1) * fb, b]

    def _ky(self):  # this rank's ky wavenumbers
        return self.kc[self.r * self.m:(self.r + 1) * self.m]

    def _kyslab(self, f):  # slot f as [N x][m ky][nkp]
        return self._c[f].view(self.N, self.m, self.nkp)

    def slab_prime(self, u):
        kx = self.kc.view(-1, 1, 1)
        for c in range(3):
            a = torch.fft.ifft(u[c], dim=0, norm="forward")
            b = torch.fft.ifft(1j * kx * u[c], dim=0, norm="forward")
            self._kyslab(c).copy_(a)
            self._kyslab(3 + c).copy_(b)

    def slab_middle(self, umax=None):
        N, m, P = self.N, self.m, self.P
        recv1 = self._c[9:9 + self.n1].view(self.n1, P, m, m, self.nkp)
        # [f][r][x_l][ky_l][kz] -> [f][x_l][y = r m + ky_l][kz]
        X = recv1.permute(0, 2, 1, 3, 4).reshape(self.n1, m, N, self.nkp)[..., : self.nk]
        ky = self.kc.view(1, -1, 1)
        kz = self.kz.view(1, 1, -1)
        iy = lambda a: torch.fft.ifft(a, dim=1, norm="forward")
        a = [iy(X[c]) for c in range(3)]
        dx = [iy(X[3 + c]) for c in range(3)]
        dy = [iy(1j * ky * X[c]) for c in range(3)]
        dz = [1j * kz * a[c] for c in range(3)]
        c2r = lambda h: torch.fft.irfft(h, n=N, dim=2, norm="forward") / float(N) ** 3
        u = [c2r(a[c]) for c in range(3)]
        A = [[c2r(dx[j]) for j in range(3)], [c2r(dy[j]) for j in range(3)], [c2r(dz[j]) for j in range(3)]]
        if umax is not None:
            self._umax_store = max(float(t.max()) for t in u)
        ox, oy, oz = A[1][2] - A[2][1], A[2][0] - A[0][2], A[0][1] - A[1][0]
        Nc = [u[1] * oz - u[2] * oy, u[2] * ox - u[0] * oz, u[0] * oy - u[1] * ox]
        dxg = 2 * math.pi / N
        ss = (A[0][0] ** 2 + 0.5 * (A[0][1] + A[1][0]) ** 2 + A[1][1] ** 2 + 0.5 * (A[0][2] + A[2][0]) ** 2
              + 0.5 * (A[1][2] + A[2][1]) ** 2 + A[2][2] ** 2)
        nut = torch.sqrt(2 * ss) * (self.cs * dxg) ** 2
        S = lambda i, j: A[i][i] if i == j else 0.5 * (A[i][j] + A[j][i])
        r2c = lambda p: torch.fft.fft(torch.fft.rfft(p, dim=2), dim=1)  # z r2c, then y forward
        out = []
        for c in range(3):
            G = r2c(Nc[c]) + 2j * (ky * r2c(S(c, 1) * nut) + kz * r2c(S(c, 2) * nut))
            out.append(G)
        for c in range(3):
            out.append(r2c(S(c, 0) * nut))
        send2 = self._c[9 + self.n1: 9 + self.n1 + self.n2].view(self.n2, P, m, m, self.nkp)
        for f, F in enumerate(out):  # [x_l][y = b m + ky_l] -> block b
            send2[f, ..., : self.nk].copy_(F.view(m, P, m, self.nk).permute(1, 0, 2, 3))
        if umax is not None:
            import struct
            bits = struct.unpack("<Q", struct.pack("<d", self._umax_store))[0]
            bits = (~bits & 0xFFFFFFFFFFFFFFFF) if (bits >> 63) else (bits | 0x8000000000000000)
            umax.fill_(bits - (1 << 64) if bits >= (1 << 63) else bits)

    def slab_stage(self, k, dt, ucur, u0, u1, uout, aux=None, flags=0):
        N = self.N
        kx = self.kc.view(-1, 1, 1)
        ky = self._ky().view(1, -1, 1)
        kz = self.kz.view(1, 1, -1)
        fx = lambda a: torch.fft.fft(a, dim=0)
        R = [fx(self._kyslab(c)[..., : self.nk]) + 2j * kx * fx(self._kyslab(3 + c)[..., : self.nk]) for c in range(3)]
        mask = (kx.abs() < self.kmax) & (ky.abs() < self.kmax) & (kz.abs() < self.kmax)
        R = [r * mask for r in R]
        K2 = kx * kx + ky * ky + kz * kz
        kk = torch.where(K2 == 0, torch.ones_like(K2), K2)
        Pj = (R[0] * kx + R[1] * ky + R[2] * kz) / kk
        K = [kx, ky, kz]
        for c in range(3):
            dU = R[c] - Pj * K[c] - self.nu * K2 * ucur[c, ..., : self.nk]
            if k == 0:
                un = u0[c, ..., : self.nk] + (0.5 * dt) * dU
            elif k == 1:
                un = u0[c, ..., : self.nk] - dt * dU + (2.0 * dt) * dU
            else:
                un = u0[c, ..., : self.nk] + dt * (dU / 6 + 2 * dU / 3 + dU / 6)
            uout[c, ..., : self.nk] = un
        if not (flags & nat.STAGE_NO_PREPARE):
            self.slab_prime(uout)

    def check(self):
        return 0
