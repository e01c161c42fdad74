"""The seeded synthetic initial fields: the package's generator
(sles.synthetic, torch on any device) against the oracle's NumPy restatement
of the same recipe, for the same seeds.  The bench's GPU arm draws its fields
from the former and its CPU arm from the latter, so they must agree.

Bar: relative L2 below 1e-12 (both draw the phases from
numpy.random.default_rng(seed); only the FFT libraries differ).
"""
import numpy as np
import pytest
import torch

from oracle import spectral_oracle as so
from sles import synthetic


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


@pytest.mark.parametrize("n,k0,seed", [(32, 4.0, 0), (32, 6.0, 3), (48, 4.0, 1), (64, 6.0, 2)])
def test_random_spectrum_matches_oracle_cpu(n, k0, seed):
    got = synthetic.random_spectrum_velocity(n, k0, 1.0, seed=seed, device="cpu")
    ref = so.random_spectrum_velocity(n, k0=k0, u0=1.0, seed=seed)
    for g, r in zip(got, ref):
        assert rel(g.numpy(), r) < 1e-12


@pytest.mark.parametrize("n,seed", [(64, 0), (128, 5)])
def test_gaussian_vorticity_matches_oracle_cpu(n, seed):
    got = synthetic.gaussian_vorticity_2d(n, seed=seed, device="cpu")
    assert rel(got.numpy(), so.gaussian_vorticity_2d(n, seed=seed)) < 1e-12


def test_taylor_green_matches_oracle_cpu():
    got = synthetic.taylor_green(16, device="cpu")
    for g, r in zip(got, so.taylor_green(16)):
        assert np.max(np.abs(g.numpy() - r)) < 1e-15


@pytest.mark.gpu
@pytest.mark.parametrize("n,k0,seed", [(64, 4.0, 0), (128, 6.0, 1)])
def test_random_spectrum_matches_oracle_gpu(n, k0, seed):
    got = synthetic.random_spectrum_velocity(n, k0, 1.0, seed=seed, device="cuda")
    ref = so.random_spectrum_velocity(n, k0=k0, u0=1.0, seed=seed)
    for g, r in zip(got, ref):
        assert rel(g.cpu().numpy(), r) < 1e-12
    torch.cuda.synchronize()
