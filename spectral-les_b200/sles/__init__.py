"""B200-native right-hand side and time stepping for the pseudo-spectral
Navier-Stokes / LES solver a-k-sangwan/spectral-LES, behind the reference's
own Python call surface.

    from sles.initialize_domain import InitializeDomain
    from sles.initial import initial_velocity, initial_vorticity
    from sles import RK4_method, RK3_method, ETD2_method
    from sles.SM_solver import spectralMethodSolver

Arithmetic runs in hand-written sm_100a CUDA kernels (libsles_b200.so) called
through a C ABI; see include/sles.h.
"""
from . import _native  # noqa: F401

__version__ = "0.1.0"
