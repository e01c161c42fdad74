"""Shared pytest setup: the ``gpu`` marker and import paths.

``-m "not gpu"`` runs the oracle-vs-golden checks, host-side logic and the
C-ABI symbol checks on CPU; ``-m gpu`` runs the CUDA parity tests.
"""
import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_ROOT = os.path.join(REPO, "spectral-les_b200")
for p in (REPO, PKG_ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def step_cases():
    """Fixtures of fixed-dt integrator runs (the others hold operator,
    diagnostic or driver-loop records)."""
    return sorted(f[:-4] for f in os.listdir(GOLDEN)
                  if f.endswith(".npz") and not f.startswith(("ops", "diag", "solver_")))


def solver_cases():
    """Fixtures of the reference's driver loop (spectralMethodSolver)."""
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.startswith("solver_") and f.endswith(".npz"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
