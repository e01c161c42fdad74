"""CPU oracle for the spectral-LES right-hand-side and time-stepping path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: it is imported by
``tests/``, by ``__graft_entry__.smoke()`` and by the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py``.  The product path
(``spectral-les_b200/sles``) never imports it and has no CPU fallback.

It is a float64 NumPy restatement, written for this project, of the
algorithm in a-k-sangwan/spectral-LES (pure Python/NumPy over mpi4py-fft).
Every function cites the reference ``file:line`` it follows.  Transform
conventions follow the reference's ``mpi4py_fft.PFFT`` call sites:
``forward(..., normalize=False)`` is an unscaled r2c along the last axis and
c2c along the others (``numpy.fft.rfftn``), ``backward(..., normalize=True)``
is the inverse scaled by 1/N^d (``numpy.fft.irfftn``); c2r discards the
imaginary part of the zero and Nyquist bins of the last axis, exactly as
pocketfft does.

Parity pin: ``tests/golden/make_golden.py`` runs the reference's own
``src/`` modules, unmodified, under a single-rank shim and stores their
outputs in ``tests/golden/*.npz``; ``tests/test_oracle_golden.py`` checks this
restatement against those fixtures to ~1e-13.

Two integrator modes are provided.  ``parity=True`` (default) reproduces the
reference exactly, including its quirks: the RK3 scheme collapses to
U0 + dt*k3 (src/RK3_method.py:26-32), ETD2 after step 1 uses the reference's
F1 coefficient and drops the LES stress (src/ETD2_method.py:16-29, 39-46).
``parity=False`` gives the corrected schemes used for the accuracy studies:
SSP-RK3 (Shu & Osher 1988) and Cox & Matthews (2002) ETD2 with the LES stress
inside the nonlinear term.
"""
from __future__ import annotations

import math
import numpy as np

__all__ = [
    "OracleDomain", "wavenumbers", "fwd", "bwd",
    "U_cross_omega", "del_cross_U", "velocity_gradient", "residue_stress",
    "nuR_smagorinsky", "nuR_vreman", "compute_rhs", "rk4_step", "rk3_step",
    "etd2_step", "step", "initial_velocity", "initial_vorticity",
    "taylor_green", "random_spectrum_velocity", "gaussian_vorticity_2d",
    "energy", "dissipation", "shell_spectrum", "reference_binned_spectrum",
    "etd2_coefficients", "set_fft_workers", "U_square", "dissipation_rate", "compute_dt",
    "solver_loop",
]

_FFT_WORKERS = None  # None -> numpy.fft (pocketfft, 1 thread); int -> scipy.fft workers


def set_fft_workers(n):
    """Use scipy.fft with ``n`` worker threads (None restores numpy.fft)."""
    global _FFT_WORKERS
    _FFT_WORKERS = n


def _axes(a, dim):
    return tuple(range(a.ndim - dim, a.ndim))


def fwd(a, dim):
    """Unscaled r2c over the last ``dim`` axes (PFFT.forward(normalize=False),
    src/math_formula.py:7-12, src/initial.py:13)."""
    if _FFT_WORKERS:
        import scipy.fft as sf
        return sf.rfftn(a, axes=_axes(a, dim), workers=_FFT_WORKERS)
    return np.fft.rfftn(a, axes=_axes(a, dim))


def bwd(a, dim, n):
    """c2r scaled by 1/n^dim (PFFT.backward(normalize=True),
    src/math_formula.py:18-24, src/RK4_method.py:41)."""
    s = (n,) * dim
    if _FFT_WORKERS:
        import scipy.fft as sf
        return sf.irfftn(a, s=s, axes=_axes(a, dim), workers=_FFT_WORKERS)
    return np.fft.irfftn(a, s=s, axes=_axes(a, dim))


def wavenumbers(n, dim):
    """Integer wavenumber grid, |k|^2, K/|k|^2 and the 2/3 cube mask.

    Follows src/initialize_domain.py:76-79 (kx = fftfreq*N, last-axis kz is the
    first N/2+1 entries with the Nyquist entry flipped to +N/2,
    kmax = 2/3*(N/2+1)), :99-114 (3D meshgrid, mask = every |K_i| < kmax),
    :144-157 (2D) and :162-165 (K2 integer, K_over_K2 with K2=0 -> 1).
    """
    kx = np.fft.fftfreq(n, 1.0 / n)
    kz = kx[: n // 2 + 1].copy()
    kz[-1] *= -1
    kmax = 2.0 / 3.0 * (n // 2 + 1)
    if dim == 3:
        K = np.array(np.meshgrid(kx, kx, kz, indexing="ij"), dtype=int)
    else:
        K = np.array(np.meshgrid(kx, kz, indexing="ij"), dtype=int)
    mask = np.ones(K.shape[1:], dtype=bool)
    for i in range(dim):
        mask &= np.abs(K[i]) < kmax
    K2 = np.sum(K * K, 0, dtype=int)
    KoK2 = K.astype(float) / np.where(K2 == 0, 1, K2).astype(float)
    return K, K2, KoK2, mask


class OracleDomain:
    """State bag mirroring ``InitializeDomain`` (src/initialize_domain.py:19-186).

    ``n`` is the computational grid.  The reference divides its
    ``No_of_gridpoint`` argument by 4 when LES is on (initialize_domain.py:38-40);
    ``from_reference_args`` applies that rule.
    """

    def __init__(self, n, dim=3, nu=0.01, dt=0.01, les_model=None, Cs=0.14,
                 method="RK4", forcing=0.0, parity=True):
        self.N = int(n)
        self.dim = int(dim)
        self.nu = float(nu)
        self.dt = float(dt)
        self.LES_ON = les_model is not None
        self.LES_model = les_model.upper() if les_model else None
        self.Cs = float(Cs)
        self.dx = 2 * math.pi / self.N                      # initialize_domain.py:42
        self.method = method
        self.forcing = float(forcing)
        self.parity = bool(parity)
        self.firstIteration = True                           # initialize_domain.py:45
        self.K, self.K2, self.K_over_K2, self.dealias = wavenumbers(self.N, self.dim)
        rshape = (self.N,) * self.dim
        cshape = self.K.shape[1:]
        self.U = np.zeros((self.dim,) + rshape)
        self.U_hat = np.zeros((self.dim,) + cshape, dtype=complex)
        self.U_hat0 = np.zeros_like(self.U_hat)
        self.U_hat1 = np.zeros_like(self.U_hat)
        self.dU = np.zeros_like(self.U_hat)
        self.F0 = np.zeros_like(self.U_hat)
        self.F1 = np.zeros_like(self.U_hat)
        self.temp_I = np.zeros_like(self.U_hat)
        self.curl = np.zeros((3,) + rshape) if self.dim == 3 else np.zeros(rshape)
        self.a = [1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0]  # initialize_domain.py:166
        self.b = [0.5, 0.5, 1.0]                                # initialize_domain.py:167

    @classmethod
    def from_reference_args(cls, No_of_gridpoint, dimension=3, nu=0.01,
                            time_stepSize=0.01, LES_ON=0, LES_model=None,
                            Cs=0.14, method="ETD2", forcing=0.0, parity=True):
        les = LES_ON == 1
        n = int(No_of_gridpoint / (4 if les else 1))         # initialize_domain.py:38-40
        return cls(n, dimension, nu, time_stepSize, LES_model if les else None,
                   Cs, method, forcing, parity)

    def grid(self):
        """Physical coordinates x_i = 2*pi*j/N (initialize_domain.py:83-88)."""
        n = self.N
        return np.mgrid[(slice(0, n),) * self.dim].astype(float) * 2 * np.pi / n


# ---------------------------------------------------------------------------
# spectral operators (src/math_formula.py)
# ---------------------------------------------------------------------------

def U_cross_omega(d, U, curl):
    """rfftn(u x omega); 2D: (v*w, -u*w).  src/math_formula.py:5-13."""
    if d.dim == 2:
        return np.array([fwd(U[1] * curl, 2), fwd(-U[0] * curl, 2)])
    return np.array([
        fwd(U[1] * curl[2] - U[2] * curl[1], 3),
        fwd(U[2] * curl[0] - U[0] * curl[2], 3),
        fwd(U[0] * curl[1] - U[1] * curl[0], 3),
    ])


def del_cross_U(d, U_hat):
    """curl = irfftn(i k x U_hat); 2D scalar.  src/math_formula.py:16-25."""
    K, n = d.K, d.N
    if d.dim == 2:
        return bwd(1j * (K[0] * U_hat[1] - K[1] * U_hat[0]), 2, n)
    c = np.empty((3,) + (n,) * 3)
    c[2] = bwd(1j * (K[0] * U_hat[1] - K[1] * U_hat[0]), 3, n)
    c[1] = bwd(1j * (K[2] * U_hat[0] - K[0] * U_hat[2]), 3, n)
    c[0] = bwd(1j * (K[1] * U_hat[2] - K[2] * U_hat[1]), 3, n)
    return c


def velocity_gradient(d, U_hat):
    """A[i][j] = d u_j / d x_i = irfftn(i K_i U_hat_j).  src/math_formula.py:27-62
    (a12 = irfftn(i K0 U_hat1) = dv/dx)."""
    n = d.N
    A = np.empty((d.dim, d.dim) + (n,) * d.dim)
    for i in range(d.dim):
        for j in range(d.dim):
            A[i, j] = bwd(1j * d.K[i] * U_hat[j], d.dim, n)
    return A


def nuR_smagorinsky(d, A):
    """nu_t = (Cs dx)^2 sqrt(2 S:S), S_ij = (a_ij + a_ji)/2.
    src/smagorinsky.py:24-47."""
    ss = np.zeros(A.shape[2:])
    for i in range(d.dim):
        ss += A[i, i] * A[i, i]
        for j in range(i + 1, d.dim):
            ss += 0.5 * (A[i, j] + A[j, i]) ** 2
    return np.sqrt(2.0 * ss) * (d.Cs * d.dx) ** 2


def nuR_vreman(d, A):
    """Vreman eddy viscosity with the reference's thresholds.

    src/vreman.py:30-123 (3D) and :124-147 (2D): with b_pq = sum_m a_mp a_mq,
    B = b11 b22 - b12^2 + b11 b33 - b13^2 + b22 b33 - b23^2 (2D: first pair),
    aa = sum a_ij^2, nu = sqrt(B) * [aa > 1e-4 and sqrt(B) > aa/1e7]
    * sqrt(1/aa) * 2.5 Cs^2 dx^2.  B is not clamped: a round-off negative B
    gives NaN, as in the reference.
    """
    dim = d.dim
    b = np.empty((dim, dim) + A.shape[2:])
    for p in range(dim):
        for q in range(dim):
            b[p, q] = sum(A[m, p] * A[m, q] for m in range(dim))
    if dim == 3:
        B = (b[0, 0] * b[1, 1] - b[0, 1] * b[0, 1]
             + b[0, 0] * b[2, 2] - b[0, 2] * b[0, 2]
             + b[1, 1] * b[2, 2] - b[1, 2] * b[1, 2])
    else:
        B = b[0, 0] * b[1, 1] - b[0, 1] * b[0, 1]
    with np.errstate(invalid="ignore", divide="ignore"):
        nu = np.sqrt(B)
        aa = np.sum(A * A, axis=(0, 1))
        gate = (aa > 10e-5) & (nu > aa / 10e6)
        nu = nu * np.where(gate, np.sqrt(1.0 / aa), 0.0) * (2.5 * d.Cs * d.Cs * d.dx * d.dx)
    return nu


def residue_stress(d, A, nuR, temp_prev=None):
    """T_hat_i = 2i * mask * sum_j K_j rfftn(nu_t S_ij).  src/math_formula.py:64-127.

    2D follows the reference literally (math_formula.py:128-146): component 0
    is written twice, the second expression wins, and component 1 keeps its
    previous content (zeros from initialize_domain.py:175).
    """
    dim, K, m = d.dim, d.K, d.dealias
    S = lambda i, j: 0.5 * (A[i, j] + A[j, i]) if i != j else A[i, i]
    if dim == 3:
        T = np.empty((3,) + K.shape[1:], dtype=complex)
        for i in range(3):
            acc = 0
            for j in range(3):
                acc = acc + K[j] * fwd(S(i, j) * nuR, 3)
            T[i] = acc * (2.0 * 1j * m)
        return T
    T = np.zeros((2,) + K.shape[1:], dtype=complex) if temp_prev is None else temp_prev.copy()
    T[0] = (K[0] * fwd(S(0, 1) * nuR, 2) + K[1] * fwd(S(1, 1) * nuR, 2)) * (2.0 * 1j * m)
    return T


def les_stress(d, U_hat):
    """Smagorinsky_model / Vreman_model (src/smagorinsky.py:8-21,
    src/vreman.py:8-21): gradients -> nu_t -> residue_stress."""
    A = velocity_gradient(d, U_hat)
    if d.LES_model[0] == "S":                               # RK4_method.py:50
        nu = nuR_smagorinsky(d, A)
    else:
        if d.dim == 2 and d.parity:
            raise AttributeError("'InitializeDomain' object has no attribute 'aTemp' "
                                 "(the reference allocates aTemp only in 3D)")
        nu = nuR_vreman(d, A)
    d.temp_I = residue_stress(d, A, nu, d.temp_I)
    return d.temp_I


def compute_rhs(d, rk, record_F1=False):
    """dU = P(mask*N_hat + T_hat) [+ f U_hat, k != 0] - nu K^2 U_hat.

    src/RK4_method.py:38-71 (== src/RK3_method.py:44-77): for rk > 0 the
    physical U and curl are recomputed from U_hat; rk == 0 reuses the stored
    ones.  When ``record_F1`` (method ETD2) F1 is the projected term before the
    viscous term and before T_hat is added back (RK4_method.py:65-66).
    """
    dim, n = d.dim, d.N
    if rk > 0:
        d.U = bwd(d.U_hat, dim, n)                         # RK4_method.py:40-43
        d.curl = del_cross_U(d, d.U_hat)                    # :44-46
    dU = U_cross_omega(d, d.U, d.curl)                      # :47
    dU *= d.dealias                                         # :48
    if d.LES_ON:
        T = les_stress(d, d.U_hat)                          # :49-51
        P = np.sum((dU + T) * d.K_over_K2, 0)               # :52-54
    else:
        T = None
        P = np.sum(dU * d.K_over_K2, 0)                     # :56
    dU -= P * d.K                                           # :57
    if d.forcing > 0.0:                                     # :58-64
        f = d.forcing * d.U_hat
        f[(slice(None),) + (0,) * dim] = 0.0
        dU += f
    if record_F1:
        d.F1 = dU.copy()                                    # :65-66
    if d.nu > 0.0:
        dU -= d.nu * d.K2 * d.U_hat                         # :67-68
    if d.LES_ON:
        dU += T                                             # :69-70
    d.dU = dU
    return dU


def _refresh_physical(d):
    d.curl = del_cross_U(d, d.U_hat)
    d.U = bwd(d.U_hat, d.dim, d.N)


def rk4_step(d):
    """Classical RK4 accumulating into U_hat1.  src/RK4_method.py:20-35.
    U_hat1 must equal U_hat on entry (the driver sets it, SM_solver.py:33)."""
    rec = d.method == "ETD2"
    d.U_hat0 = d.U_hat.copy()
    for rk in range(4):
        dU = compute_rhs(d, rk, record_F1=rec)
        if rk < 3:
            d.U_hat = d.U_hat0 + d.b[rk] * d.dt * dU
        d.U_hat1 = d.U_hat1 + d.a[rk] * d.dt * dU
    d.U_hat = d.U_hat1.copy()
    _refresh_physical(d)


def rk3_step(d):
    """Reference RK3 (src/RK3_method.py:20-41); with one dU buffer it reduces
    to U0 + dt*k3.  parity=False: SSP-RK3 (Shu & Osher 1988)."""
    dt = d.dt
    U0 = d.U_hat.copy()
    d.U_hat0 = U0
    if d.parity:
        dU = compute_rhs(d, 0)
        d.U_hat = U0 + 0.5 * dt * dU
        dU = compute_rhs(d, 1)
        d.U_hat = U0 - dt * dU + 2.0 * dt * dU
        dU = compute_rhs(d, 2)
        d.U_hat = U0 + dt * (1 / 6 * dU + 2 / 3 * dU + 1 / 6 * dU)
    else:
        dU = compute_rhs(d, 0)
        d.U_hat = U0 + dt * dU
        dU = compute_rhs(d, 1)
        d.U_hat = 0.75 * U0 + 0.25 * (d.U_hat + dt * dU)
        dU = compute_rhs(d, 2)
        d.U_hat = (1.0 / 3.0) * U0 + (2.0 / 3.0) * (d.U_hat + dt * dU)
    _refresh_physical(d)


def etd2_coefficients(K2, nu, dt, parity):
    """Integrating-factor and ETD2 weights per |k|^2 (float64).

    parity: the reference's weights (src/ETD2_method.py:16-29):
      c1 = (1 + h L)/(h L^2), c0 = (1 - e^{-hL} - hL)/(h L^2), 1 and 0 at K2 == 0.
    corrected (Cox & Matthews 2002, eq. 22 with c = -L):
      c1 = ((1 - z) e^{-z} - 1 + 2 z)/(h L^2),  c0 = (-e^{-z} + 1 - z)/(h L^2),
    z = h L = dt nu K2; for |z| < 1e-2 the Taylor series
      c1 = h (3/2 - 2z/3 + z^2/4 - z^3/15),  c0 = h (-1/2 + z/6 - z^2/24 + z^3/120)
    avoids cancellation (limits 3h/2 and -h/2 at z -> 0).
    """
    h = dt
    L = nu * K2.astype(float)
    z = h * L
    E = np.exp(-z)
    if parity:
        den = np.where(K2 == 0, 1.0, h * L * L)
        c1 = (1.0 - z + 2.0 * z) / den
        c0 = (-E + 1.0 - z) / den
        return E, c1, c0
    with np.errstate(divide="ignore", invalid="ignore"):
        zz = np.where(z == 0, 1.0, z)
        c1 = h * ((1.0 - zz) * np.exp(-zz) - 1.0 + 2.0 * zz) / (zz * zz)
        c0 = h * (-np.exp(-zz) + 1.0 - zz) / (zz * zz)
    small = np.abs(z) < 1e-2
    c1s = h * (1.5 - 2.0 * z / 3.0 + z * z / 4.0 - z ** 3 / 15.0)
    c0s = h * (-0.5 + z / 6.0 - z * z / 24.0 + z ** 3 / 120.0)
    return E, np.where(small, c1s, c1), np.where(small, c0s, c0)


def _nonlinear_projected(d, with_les):
    """P(mask * N_hat [+ T_hat]) (src/ETD2_method.py:39-46 without LES)."""
    N = U_cross_omega(d, d.U, d.curl) * d.dealias
    if with_les:
        N = N + les_stress(d, d.U_hat)
    P = np.sum(N * d.K_over_K2, 0)
    return N - P * d.K


def _explicit_term(d, with_les):
    """The explicit part of the corrected ETD2 scheme: P(mask N_hat [+ T_hat])
    plus the linear forcing f U_hat on k != 0, added after the projection as
    computeRHS adds it (src/RK4_method.py:58-64).  The reference's ETD2
    forcing branch (src/ETD2_method.py:47-56) cannot run (it reads an unset
    domain.epsilon); this follows the Cox-Matthews scheme with the forcing
    treated explicitly."""
    F = _nonlinear_projected(d, with_les)
    if d.forcing > 0.0:
        f = d.forcing * d.U_hat
        f[(slice(None),) + (0,) * d.dim] = 0.0
        F = F + f
    return F


def etd2_step(d):
    """src/ETD2_method.py:7-37.  Step 1 is RK4 (recording F1, parity) ; later
    steps advance with the exponential integrator."""
    if d.firstIteration:
        if d.parity:
            rk4_step(d)
        else:
            d.F1 = _explicit_term(d, d.LES_ON)
            d.method, m = "RK4", d.method
            rk4_step(d)
            d.method = m
        d.firstIteration = False
        return
    if d.forcing > 0.0 and d.parity:
        # src/ETD2_method.py:47-50 reads domain.epsilon, which is never set
        raise AttributeError("'InitializeDomain' object has no attribute 'epsilon'")
    d.F0 = d.F1
    # parity: the reference evaluates u x omega only here (src/ETD2_method.py:39-46)
    d.F1 = _nonlinear_projected(d, with_les=False) if d.parity else _explicit_term(d, d.LES_ON)
    E, c1, c0 = etd2_coefficients(d.K2, d.nu, d.dt, d.parity)
    if d.parity:
        d.U_hat = d.U_hat * E
        d.U_hat = d.U_hat + (d.F1 * (1.0 - d.dt * d.nu * d.K2 + 2 * d.dt * d.nu * d.K2)
                             + d.F0 * (-E + 1 - d.dt * d.nu * d.K2)) / \
            np.where(d.K2 == 0, 1, d.dt * (d.nu * d.K2) ** 2)
    else:
        d.U_hat = d.U_hat * E + d.F1 * c1 + d.F0 * c0
    d.U = bwd(d.U_hat, d.dim, d.N)
    d.curl = del_cross_U(d, d.U_hat)


def step(d):
    """Dispatch as src/SM_solver.py:52-59."""
    if d.method == "RK4":
        rk4_step(d)
    elif d.method == "ETD2":
        etd2_step(d)
    elif d.method == "RK3":
        rk3_step(d)
    else:
        raise ValueError("Invalid method name")


# ---------------------------------------------------------------------------
# initial conditions (src/initial.py) and synthetic fields
# ---------------------------------------------------------------------------

def initial_velocity(d, u, v, w=None):
    """src/initial.py:7-18: U = given arrays, U_hat = rfftn(U), curl from U_hat."""
    U = [u, v] + ([w] if d.dim == 3 else [])
    d.U = np.array([np.broadcast_to(np.asarray(x, float), (d.N,) * d.dim) for x in U])
    d.U_hat = fwd(d.U, d.dim)
    d.curl = del_cross_U(d, d.U_hat)


def initial_vorticity(d, omega):
    """src/initial.py:39-54: streamfunction phi = omega_hat/K2 (phi(0)=0),
    U_hat = (i ky phi, -i kx phi); curl keeps the given omega."""
    phi = fwd(np.asarray(omega, float), d.dim) / np.where(d.K2 == 0, 1, d.K2).astype(float)
    phi[(0,) * d.dim] = 0
    d.U_hat = np.zeros_like(d.U_hat)
    d.U_hat[0] = 1j * d.K[1] * phi
    d.U_hat[1] = -1j * d.K[0] * phi
    if d.dim == 3:
        d.U_hat[2] = 0
        d.curl[2] = omega
    else:
        d.curl = np.array(omega, float)
    d.U = bwd(d.U_hat, d.dim, d.N)


def taylor_green(n):
    """u = sin x cos y cos z, v = -cos x sin y cos z, w = 0 on x_i = 2 pi j/N."""
    X = np.mgrid[:n, :n, :n].astype(float) * 2 * np.pi / n
    u = np.sin(X[0]) * np.cos(X[1]) * np.cos(X[2])
    v = -np.cos(X[0]) * np.sin(X[1]) * np.cos(X[2])
    return u, v, np.zeros_like(u)


def _model_spectrum(k, k0, u0):
    return 16.0 * math.sqrt(2.0 / math.pi) * u0 * u0 * k ** 4 / k0 ** 5 * np.exp(-2.0 * k * k / (k0 * k0))


def random_spectrum_velocity(n, k0=4.0, u0=1.0, seed=0):
    """Solenoidal random-phase velocity with E(k) = 16 sqrt(2/pi) u0^2 k^4/k0^5
    exp(-2 k^2/k0^2) (no counterpart in the reference).

    Per rfft mode with k != 0 inside the 2/3 cube and off the Nyquist planes:
    |u_hat_c| = sqrt(E(|k|)/(2 pi |k|^2)), phase_c ~ U[0, 2 pi) from
    ``numpy.random.default_rng(seed)``; project out k (k . u_hat); rescale each
    integer shell so that sum 1/2 |u_hat|^2 (weights 2 for 0 < kz < N/2) equals
    E(k); physical field = irfftn(u_hat) * N^3 (real by construction).
    """
    K, K2, _, mask = wavenumbers(n, 3)
    rng = np.random.default_rng(seed)
    kmag = np.sqrt(K2.astype(float))
    nyq = (np.abs(K[0]) == n // 2) | (np.abs(K[1]) == n // 2) | (np.abs(K[2]) == n // 2)
    live = mask & (K2 > 0) & ~nyq
    amp = np.zeros_like(kmag)
    amp[live] = np.sqrt(_model_spectrum(kmag[live], k0, u0) / (2 * np.pi * kmag[live] ** 2))
    phase = rng.uniform(0.0, 2 * np.pi, size=(3,) + kmag.shape)
    uh = amp[None] * np.exp(1j * phase)
    # make the kz = 0 plane Hermitian (what a real field's rfftn holds)
    uh = np.fft.rfftn(np.fft.irfftn(uh, s=(n, n, n), axes=(1, 2, 3)), axes=(1, 2, 3))
    kk = np.where(K2 == 0, 1, K2).astype(float)
    kdotu = np.sum(K * uh, 0)
    uh = uh - K * kdotu / kk
    uh[:, ~live] = 0.0
    w = np.where((K[2] > 0) & (K[2] < n // 2), 2.0, 1.0)
    shell = np.rint(kmag).astype(int)
    e_mode = 0.5 * np.sum(np.abs(uh) ** 2, 0) * w
    e_shell = np.bincount(shell.ravel(), weights=e_mode.ravel())
    target = _model_spectrum(np.arange(e_shell.size, dtype=float), k0, u0)
    scale = np.where(e_shell > 0, np.sqrt(target / np.where(e_shell > 0, e_shell, 1)), 0.0)
    uh = uh * scale[shell][None]
    u = np.fft.irfftn(uh, s=(n, n, n), axes=(1, 2, 3)) * n ** 3
    return u[0], u[1], u[2]


def gaussian_vorticity_2d(n, seed=0, kp=10.0):
    """2D Gaussian random vorticity with spectrum (k/kp)^2 exp(-(k/kp)^2),
    zero mean, rms 1 (no counterpart in the reference)."""
    K, K2, _, _ = wavenumbers(n, 2)
    rng = np.random.default_rng(seed)
    k = np.sqrt(K2.astype(float))
    shape = K2.shape
    g = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    wh = g * (k / kp) ** 2 * np.exp(-(k / kp) ** 2)
    nyq = (np.abs(K[0]) == n // 2) | (np.abs(K[1]) == n // 2)
    wh[nyq] = 0.0
    wh[0, 0] = 0.0
    w = np.fft.irfftn(wh, s=(n, n), axes=(0, 1))
    w -= w.mean()
    return w / np.sqrt(np.mean(w * w))


# ---------------------------------------------------------------------------
# diagnostics
# ---------------------------------------------------------------------------

def _hermitian_weights(d):
    kz = d.K[-1]
    n = d.N
    return np.where((kz != 0) & (np.abs(kz) != n // 2), 2.0, 1.0)


def energy(d, U_hat=None):
    """E = 1/2 <u.u> from U_hat (Parseval, half-complex weights)."""
    Uh = d.U_hat if U_hat is None else U_hat
    w = _hermitian_weights(d)
    return 0.5 * float(np.sum(w * np.sum(np.abs(Uh) ** 2, 0))) / float(d.N) ** (2 * d.dim)


def dissipation(d, U_hat=None):
    """eps = nu <|grad u|^2> = nu sum k^2 |u_hat|^2 / N^(2d) (= 2 nu <S:S> for
    solenoidal periodic fields)."""
    Uh = d.U_hat if U_hat is None else U_hat
    w = _hermitian_weights(d)
    return d.nu * float(np.sum(w * d.K2 * np.sum(np.abs(Uh) ** 2, 0))) / float(d.N) ** (2 * d.dim)


def shell_spectrum(d, U_hat=None):
    """E(k) on integer shells round(|k|): 1/2 sum |u_hat|^2 / N^(2d), weights
    2 for 0 < kz < N/2."""
    Uh = d.U_hat if U_hat is None else U_hat
    w = _hermitian_weights(d)
    e = 0.5 * w * np.sum(np.abs(Uh) ** 2, 0) / float(d.N) ** (2 * d.dim)
    shell = np.rint(np.sqrt(d.K2.astype(float))).astype(int)
    return np.bincount(shell.ravel(), weights=e.ravel())


def reference_binned_spectrum(d, U_hat=None):
    """The reference's E(k) diagnostic: shells of width 5 in |k|, *mean* of
    sum_i |U_hat_i|^2 over the modes of a shell, x2 for kz > 0 on rank 0.
    src/SM_solver.py:94-112 (bins) and :154-192 (values)."""
    Uh = d.U_hat if U_hat is None else U_hat
    avg = 5
    k2u = np.unique(d.K2)
    ns = int(round(math.sqrt(np.max(k2u)))) // avg
    Ek = np.sum(np.abs(Uh) ** 2, 0)
    Ek = Ek.copy()
    if d.dim == 2:
        Ek[:, 1:] *= 2
    else:
        Ek[:, :, 1:] *= 2
    tk = np.zeros(ns + 1)
    tE = np.zeros(ns + 1)
    for i in range(ns + 1):
        lo, hi = (i * avg) ** 2, ((i + 1) * avg) ** 2
        if np.any(k2u[(k2u >= lo) & (k2u < hi)]):
            sel = (d.K2 >= lo) & (d.K2 < hi)
            tk[i] = np.mean(np.sqrt(d.K2[sel]))
            tE[i] = np.mean(Ek[sel])
    return tk, tE


def U_square(d):
    """sum_i mean(u_i^2) over the physical field (no 1/2): src/RK4_method.py:77-84."""
    U = np.array([bwd(d.U_hat[i], d.dim, d.N) for i in range(d.dim)])
    return float(np.sum(U * U)) / float(d.N) ** d.dim


def dissipation_rate(d):
    """nu * sum_i sum_x u_i irfftn(K^2 U_hat_i) (a sum, not a mean):
    src/RK4_method.py:87-101."""
    eps = 0.0
    for i in range(d.dim):
        u = bwd(d.U_hat[i], d.dim, d.N)
        eps += d.nu * float(np.sum(u * bwd(d.U_hat[i] * d.K2, d.dim, d.N)))
    return eps


# ---------------------------------------------------------------------------
# driver loop (src/SM_solver.py)
# ---------------------------------------------------------------------------

def compute_dt(u_max, nu, dx, CFL):
    """dt = min(CFL dx/u_max, 0.1 dx^2/nu); the reference exits below 1e-6
    (src/SM_solver.py:258-277).  Raises SystemExit there."""
    dt1 = CFL * dx / u_max
    dt2 = 0.1 * dx ** 2 / nu if nu > 0 else 1e6
    dt = min(dt1, dt2)
    if dt < 1e-6:
        raise SystemExit(1)
    return dt


def solver_loop(d, final_time, CFL=0.5, No_Ek_plot=5):
    """The loop of spectralMethodSolver (src/SM_solver.py:18-83) without file
    output: u_max = max over components and points of U (signed,
    find_max_velocity :245-255), dt from compute_dt with CFL 0.3 before the
    first step, t starts at dt_0, E(k) snapshots (width-5 bins) whenever
    t >= the next multiple of final_time/No_Ek_plot, stop at t >= final_time
    or dt < 1e-8, NaN stop.  Returns (steps, dt list, u_max list, snapshots)
    with snapshots = [(t, temp_k, temp_Ek)]."""
    dts, umaxs, snaps = [], [], []

    def umax():
        return float(np.max(d.U))  # the stored physical velocity, as the reference reads domain.U

    u = umax()
    d.dt = compute_dt(u, d.nu, d.dx, 0.3)
    dts.append(d.dt)
    umaxs.append(u)
    t = d.dt
    interval = final_time / No_Ek_plot if No_Ek_plot != 0 else 0
    counter_t = 0.0
    d.U_hat1 = d.U_hat.copy()
    steps = 0
    while True:
        if interval > 0 and t >= counter_t:
            tk, tE = reference_binned_spectrum(d)
            snaps.append((t, tk, tE))
            counter_t += interval
        if t >= final_time or d.dt < 1e-8:
            break
        t += d.dt
        step(d)
        steps += 1
        u = umax()
        d.dt = compute_dt(u, d.nu, d.dx, CFL)
        dts.append(d.dt)
        umaxs.append(u)
        if d.dt != d.dt:
            break
    return steps, dts, umaxs, snaps
