"""sles_rhs_static_workspace: the fused RHS without any device allocation.

Some callers cannot call cudaMalloc: code running where device allocation is
off limits (inside an allocator or a host application that owns every device
allocation through its own pool, or a latency-critical loop that must avoid
cudaMalloc's implicit synchronization).  For them the library exposes one entry
point whose scratch is a fixed-size device array inside the library instead of
a caller-provided workspace.  This test calls it through the C ABI and checks
it against sles_rhs (which uses the plan's workspace) on two calls in a row,
that a plan whose workspace would not fit the array is refused, and that a
bounded wait that gives up on the array's error word is reported by
sles_static_workspace_check.

Collected last (tests/test_zz_*) so that a run stopping at the first failure
has already run every other test; it also passes when run alone.
"""
import ctypes

import pytest
import torch

from sles import _native as nat
from sles.initial import initial_velocity
from sles.initialize_domain import InitializeDomain
from sles.synthetic import random_spectrum_velocity

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def _call_static(d, du):
    L = nat.load_library()
    return L.sles_rhs_static_workspace(d._plan.h, nat.ptr(d._s_uhat), None, None, nat.ptr(du), None,
                                       nat.stream_handle(d.device))


@pytest.mark.parametrize("dtype,tol", [("float32", 1e-6), ("float64", 1e-13)])
def test_static_workspace_rhs_matches_workspace_rhs(dtype, tol):
    n = 64
    d = InitializeDomain(nu=1e-3, dimension=3, time_stepSize=1e-3, No_of_gridpoint=4 * n, method="RK4",
                         LES_ON=1, LES_model="Smagorinsky", Cs=0.17, dtype=dtype)
    initial_velocity(d, *random_spectrum_velocity(n, 4.0, 1.0, seed=11))
    ref = d._new_hc(3)
    d._plan.rhs(d._s_uhat, ref)
    L = nat.load_library()
    for _ in range(2):  # two calls in a row share (and reuse) the static array
        du = d._new_hc(3)
        assert _call_static(d, du) == 0
        w = ctypes.c_uint(1)
        assert L.sles_static_workspace_check(ctypes.byref(w), nat.stream_handle(d.device)) == 0
        assert w.value == 0
        assert _rel(du[..., : d._nk], ref[..., : d._nk]) < tol


def test_static_workspace_rejects_plans_that_do_not_fit():
    n = 128  # 3D LES float32 at 128^3 needs ~80 MB of scratch, above the 32 MiB array
    d = InitializeDomain(nu=1e-3, dimension=3, time_stepSize=1e-3, No_of_gridpoint=4 * n, method="RK4",
                         LES_ON=1, LES_model="Smagorinsky", Cs=0.17, dtype="float32")
    du = d._new_hc(3)
    assert _call_static(d, du) == 4  # SLES_ERR_WORKSPACE, nothing launched


def test_static_workspace_wait_timeout_is_reported():
    """The static array's error word is read (and cleared) by
    sles_static_workspace_check: a short bounded wait on it that runs out
    comes back as SLES_ERR_TIMEOUT, and the context stays usable."""
    L = nat.load_library()
    st = nat.stream_handle(torch.device("cuda", torch.cuda.current_device()))
    w = ctypes.c_uint(0)
    assert L.sles_static_workspace_check(ctypes.byref(w), st) == 0
    assert L.sles_static_workspace_selftest_timeout(st) == 0
    assert L.sles_static_workspace_check(ctypes.byref(w), st) == 5  # SLES_ERR_TIMEOUT
    assert w.value != 0
    assert L.sles_static_workspace_check(ctypes.byref(w), st) == 0  # cleared
    test_static_workspace_rhs_matches_workspace_rhs("float32", 1e-6)
