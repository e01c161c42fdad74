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


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
