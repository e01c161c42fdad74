"""Simulation domain: the drop-in counterpart of the reference's
``InitializeDomain`` (src/initialize_domain.py:19-186).

Same constructor arguments and the same public attributes.  Differences that
follow from running on one B200:

* state lives on the GPU as torch tensors; ``U_hat``, ``U_hat0``, ``U_hat1``,
  ``F0``, ``F1`` and ``dU`` are views with the reference's shapes
  ``(dim, N, N, N//2+1)`` (3D) / ``(dim, N, N//2+1)`` (2D) of row-padded
  storage (rows padded to a multiple of 4 complex values for aligned access);
* ``U`` and ``curl`` are materialized from ``U_hat`` on first access after a
  step (the fused steppers never need them in memory);
* wavenumber arrays (``K``, ``K2``, ``K_over_K2``, ``dealias``) and the grid
  ``X`` are NumPy arrays built on first access, as in the reference; the GPU
  kernels generate wavenumbers from indices instead of reading them;
* ``fft`` is a GPU transform object with PFFT's ``forward``/``backward``
  signatures; ``comm`` is a single-rank communicator.
* extra keyword-only options: ``dtype`` ("float64" default, or "float32"),
  ``parity_mode`` (True: the reference's arithmetic including its RK3/ETD2
  quirks; False: corrected schemes), ``device``.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _native as nat
from . import autotune

__all__ = ["InitializeDomain"]

_SIZES_3D = (16, 24, 32, 48, 64, 96, 128, 256, 512)
_SIZES_2D = (16, 24, 32, 48, 64, 96, 128, 256, 512, 1024)


class _SingleRankComm:
    """Stand-in for MPI.COMM_WORLD on one GPU (Get_size/Get_rank/Allreduce)."""
    rank = 0

    def Get_size(self):
        return 1

    def Get_rank(self):
        return 0

    def Allreduce(self, send, recv, op=None):
        s = send[0] if isinstance(send, (list, tuple)) else send
        r = recv[0] if isinstance(recv, (list, tuple)) else recv
        np.asarray(r).reshape(-1)[0] = np.asarray(s).reshape(-1)[0]


class _GpuFFT:
    """PFFT-compatible transforms on the GPU (forward: unscaled r2c over all
    axes; backward: c2r scaled by 1/N^d), used by the math_formula helpers."""

    def __init__(self, domain):
        self._d = domain

    def forward(self, a, out=None, normalize=False):
        d = self._d
        x = d._as_real(a)
        nf = x.numel() // d._rsize
        hc = d._new_hc(nf)
        d._plan.fft_r2c(x, hc, nf)
        r = d._hc_view(hc).reshape(tuple(x.shape[:-d.dim]) + d._hc_shape)
        if normalize:
            r = r / float(d.N ** d.dim)
        if out is not None:
            out[...] = r
            return out
        return r

    def backward(self, a, out=None, normalize=True):
        d = self._d
        hc = d._as_hc(a)
        nf = hc.shape[0]
        r = torch.empty((nf,) + d.shape, dtype=d._rdtype, device=d.device)
        d._plan.fft_c2r(hc, r, nf)
        d._primed = None
        shp = tuple(a.shape[:-d.dim]) + d.shape
        r = r.reshape(shp)
        if not normalize:
            r = r * float(d.N ** d.dim)
        if out is not None:
            out[...] = r
            return out
        return r


class InitializeDomain:
    def __init__(self, nu: float = 0.01, final_time: float = 0.0, dimension: int = 3,
                 time_stepSize: float = 0.01, No_of_gridpoint: int = 128, forcing=0.0,
                 forcing_range=[0, 1], method="ETD2", LES_ON=0, CFL: float = 0.5,
                 Cs: float = 0.14, LES_model=None, *, dtype="float64", parity_mode=True,
                 device="cuda"):
        # scalar attributes: initialize_domain.py:34-58
        self.nu = nu
        self.CFL = CFL
        self.T = final_time
        self.dt = time_stepSize
        self.LES_ON = True if LES_ON == 1 else False
        self.NN = 4 if self.LES_ON else 1
        self.N = int(No_of_gridpoint / self.NN)
        self.N_full = No_of_gridpoint if self.LES_ON else None
        self.dx = 2 * math.pi / self.N
        self.method = method
        self.firstIteration = True
        self.forcing = forcing
        self.forcing_range = forcing_range
        self.comm = _SingleRankComm()
        self.num_processes = 1
        self.rank = 0
        self.Np = self.N
        self.dim = dimension
        self.shape = tuple(self.N for _ in range(self.dim))
        self.kx = np.fft.fftfreq(self.N, 1.0 / self.N)   # :76-79
        self.kz = self.kx[: (self.N // 2 + 1)].copy()
        self.kz[-1] *= -1
        self.kmax_dealias = 2.0 / 3.0 * (self.N // 2 + 1)
        self.a = [1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0]  # :166-167
        self.b = [0.5, 0.5, 1.0]
        self.parity_mode = bool(parity_mode)
        if self.LES_ON:
            if LES_model is None:  # :169-171 (the reference prints and exits)
                raise SystemExit("\n Please choose LES_model (Smagorinsky or Vreman)")
            self.LES_model = LES_model.upper()
            self.Cs = Cs
        else:
            self.LES_model = None
            self.Cs = Cs
        if self.dim not in (2, 3):
            raise ValueError("dimension must be 2 or 3")
        sizes = _SIZES_3D if self.dim == 3 else _SIZES_2D
        if self.N not in sizes:
            raise ValueError("grid N=%d is not compiled for dimension %d (supported: %s)"
                             % (self.N, self.dim, sizes))
        if method not in ("RK4", "RK3", "ETD2"):
            raise ValueError("Invalid method name")
        self.device = torch.device(device)
        self._rdtype = {"float64": torch.float64, "float32": torch.float32,
                        torch.float64: torch.float64, torch.float32: torch.float32}[dtype]
        self._cdtype = torch.complex128 if self._rdtype == torch.float64 else torch.complex64
        les = nat.LES_NONE
        if self.LES_ON:
            les = nat.LES_SMAGORINSKY if self.LES_model[0] == "S" else nat.LES_VREMAN  # RK4_method.py:50
        scheme = {"RK4": nat.SCHEME_RK4, "RK3": nat.SCHEME_RK3, "ETD2": nat.SCHEME_ETD2}[method]
        self._plan = nat.Plan(self.dim, self.N, self._rdtype, les, scheme, self.parity_mode, nu, Cs,
                              forcing, self.device)
        autotune.apply_cached(self._plan, method)  # kernel variants recorded by sles.autotune.tune
        self._nk, self._nkp = self._plan.nk, self._plan.nkp
        self._hc_shape = self.shape[:-1] + (self._nk,)
        self._hc_pshape = self.shape[:-1] + (self._nkp,)
        self._rsize = int(np.prod(self.shape))
        self.fft = _GpuFFT(self)
        # state storage (padded); roles are swapped instead of copying
        self._s_uhat = self._new_hc(self.dim)
        self._s_u0 = self._new_hc(self.dim)
        self._s_u1 = self._new_hc(self.dim)
        self._s_f0 = self._new_hc(self.dim) if method == "ETD2" else None
        self._s_f1 = self._new_hc(self.dim) if method == "ETD2" else None
        self._s_du = None
        self._U = torch.zeros((self.dim,) + self.shape, dtype=self._rdtype, device=self.device)
        self._curl = torch.zeros(((3,) if self.dim == 3 else ()) + self.shape, dtype=self._rdtype,
                                 device=self.device)
        self._phys_fresh = True        # U/curl match U_hat (all zeros here)
        self._phys_user = False        # U/curl were set by a setter: stage 0 must use them
        self._phys_ver = (self._U._version, self._curl._version)
        self._primed = None            # (storage data_ptr, version) whose x-inverse sits in the workspace
        self._dtctl = None             # device-side dt controller (SM_solver device mode), else None
        self._parity = 0               # step index mod 2 (the controller's u_max slot)
        self._lazy = {}

    # ------------------------------------------------------------------ storage
    def _new_hc(self, nf):
        return torch.zeros((nf,) + self._hc_pshape, dtype=self._cdtype, device=self.device)

    def _hc_view(self, s):
        return s[..., : self._nk]

    def _as_real(self, a):
        t = torch.as_tensor(a, device=self.device)
        if t.dtype != self._rdtype:
            t = t.to(self._rdtype)
        if t.shape[-self.dim:] != self.shape:
            t = torch.broadcast_to(t, t.shape[:-self.dim] + self.shape) if t.dim() >= self.dim else \
                torch.broadcast_to(t, self.shape)
        return t.contiguous()

    def _as_hc(self, a):
        """Copy (nf, ...hc shape) or a padded storage into fresh padded storage."""
        t = torch.as_tensor(a, device=self.device)
        if t.dtype != self._cdtype:
            t = t.to(self._cdtype)
        lead = t.shape[: t.dim() - self.dim]
        nf = int(np.prod(lead)) if len(lead) else 1
        t = t.reshape((nf,) + tuple(t.shape[-self.dim:]))
        s = self._new_hc(nf)
        s[..., : t.shape[-1]].copy_(t[..., : self._nk])
        return s

    # ------------------------------------------------------------ state views
    @property
    def U_hat(self):
        return self._hc_view(self._s_uhat)

    @U_hat.setter
    def U_hat(self, value):
        self.U_hat[...] = torch.as_tensor(value, device=self.device).to(self._cdtype)

    @property
    def U_hat0(self):
        return self._hc_view(self._s_u0)

    @U_hat0.setter
    def U_hat0(self, value):
        self.U_hat0[...] = torch.as_tensor(value, device=self.device).to(self._cdtype)

    @property
    def U_hat1(self):
        return self._hc_view(self._s_u1)

    @U_hat1.setter
    def U_hat1(self, value):
        self.U_hat1[...] = torch.as_tensor(value, device=self.device).to(self._cdtype)

    @property
    def F0(self):
        return None if self._s_f0 is None else self._hc_view(self._s_f0)

    @property
    def F1(self):
        return None if self._s_f1 is None else self._hc_view(self._s_f1)

    @property
    def dU(self):
        """RHS buffer written by ``computeRHS`` (the fused steppers do not
        materialize the per-stage right-hand side)."""
        if self._s_du is None:
            self._s_du = self._new_hc(self.dim)
        return self._hc_view(self._s_du)

    @property
    def U(self):
        self._ensure_phys()
        return self._U

    @U.setter
    def U(self, value):
        self._U[...] = self._as_real(value)

    @property
    def curl(self):
        self._ensure_phys()
        return self._curl

    @curl.setter
    def curl(self, value):
        self._curl[...] = self._as_real(value)

    def _ensure_phys(self):
        if not self._phys_fresh:
            self._plan.velocity_curl(self._s_uhat, self._U, self._curl)
            self._primed = None
            self._phys_fresh = True
            self._phys_user = False
            self._phys_ver = (self._U._version, self._curl._version)

    def _phys_override(self):
        """(U, curl) to use at stage 0 instead of the ones implied by U_hat, or
        (None, None).  The reference's stage 0 reuses the stored U and curl
        (src/RK4_method.py:39-47); they differ from U_hat's only after a setter
        or an in-place edit by the caller."""
        if not self._phys_fresh:
            return None, None
        edited = (self._U._version, self._curl._version) != self._phys_ver
        if self._phys_user or edited:
            return self._U, self._curl
        return None, None

    def _mark_stepped(self):
        self._phys_fresh = False
        self._phys_user = False

    # ------------------------------------------------------ reference arrays
    def _lazy_get(self, name, fn):
        if name not in self._lazy:
            self._lazy[name] = fn()
        return self._lazy[name]

    @property
    def K(self):
        def mk():
            if self.dim == 3:
                return np.array(np.meshgrid(self.kx, self.kx, self.kz, indexing="ij"), dtype=int)
            return np.array(np.meshgrid(self.kx, self.kz, indexing="ij"), dtype=int)
        return self._lazy_get("K", mk)

    @property
    def K2(self):
        return self._lazy_get("K2", lambda: np.sum(self.K * self.K, 0, dtype=int))

    @property
    def K_over_K2(self):
        return self._lazy_get("KoK2", lambda: self.K.astype(float) /
                              np.where(self.K2 == 0, 1, self.K2).astype(float))

    @property
    def dealias(self):
        def mk():
            m = np.ones(self.K.shape[1:], dtype=bool)
            for i in range(self.dim):
                m &= np.abs(self.K[i]) < self.kmax_dealias
            return m
        return self._lazy_get("dealias", mk)

    @property
    def X(self):
        return self._lazy_get("X", lambda: np.mgrid[(slice(0, self.N),) * self.dim].astype(float)
                              * 2 * np.pi / self.N)

    @property
    def d(self):
        return tuple(np.arange(s, dtype=float) * 2 * np.pi / s for s in self.shape)

    # -------------------------------------------------------------- misc
    def synchronize(self):
        torch.cuda.synchronize(self.device)
