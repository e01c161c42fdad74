"""Own r2c/c2r transforms against numpy.fft (float64 to 1e-13, float32 to 2e-6)."""
import numpy as np
import pytest
import torch

from sles.initialize_domain import InitializeDomain

pytestmark = pytest.mark.gpu

CASES3 = [16, 24, 32, 48, 64, 96, 128, 256]
CASES2 = [16, 32, 96, 256, 1024]


def _dom(n, dim, dtype):
    return InitializeDomain(No_of_gridpoint=n, dimension=dim, method="RK4", dtype=dtype)


def rel(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


@pytest.mark.parametrize("dtype,tol", [("float64", 1e-13), ("float32", 3e-6)])
@pytest.mark.parametrize("dim,n", [(3, n) for n in CASES3] + [(2, n) for n in CASES2])
def test_r2c_c2r_match_numpy(dim, n, dtype, tol):
    d = _dom(n, dim, dtype)
    rng = np.random.default_rng(n)
    x = rng.standard_normal((2,) + (n,) * dim)
    X = d.fft.forward(torch.as_tensor(x, device="cuda"))
    ref = np.fft.rfftn(x, axes=tuple(range(1, dim + 1)))
    assert rel(X.cpu().numpy(), ref) < tol
    # c2r of a non-Hermitian spectrum: imaginary parts of the kz=0/N/2 bins are
    # discarded after the c2c axes, as numpy.fft.irfftn does
    Y = ref + 0.3j * rng.standard_normal(ref.shape)
    y = d.fft.backward(torch.as_tensor(Y, device="cuda"))
    yref = np.fft.irfftn(Y, s=(n,) * dim, axes=tuple(range(1, dim + 1)))
    assert rel(y.cpu().numpy(), yref) < tol
