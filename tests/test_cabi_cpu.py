"""C-ABI checks that need no GPU: the library loads, exports every entry point
declared in include/sles.h, and validates plan descriptors on the host."""
import ctypes
import os
import re

import pytest

from conftest import REPO
from sles import _native as nat

HEADER = os.path.join(REPO, "include", "sles.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|const char\*)\s+(sles_\w+)\s*\(", txt, re.M)))


def test_header_and_binding_agree():
    assert declared() == sorted(nat.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(nat.LIB_PATH)
    for name in declared():
        assert hasattr(lib, name), name


def _desc(**kw):
    base = dict(dim=3, n=64, dtype=nat.SLES_F32, les_model=nat.LES_SMAGORINSKY, scheme=nat.SCHEME_RK3,
                parity=1, nu=1e-4, cs=0.17, forcing=0.0)
    base.update(kw)
    return nat.PlanDesc(**base)


def test_plan_create_layout_destroy_on_host():
    L = nat.load_library()
    h = ctypes.c_void_p()
    d = _desc()
    assert L.sles_plan_create(ctypes.byref(d), ctypes.byref(h)) == 0
    lay = nat.Layout()
    assert L.sles_plan_layout(h, ctypes.byref(lay)) == 0
    assert lay.nk == 33 and lay.nkp == 36 and lay.hc_elems == 64 * 64 * 36 and lay.real_elems == 64 ** 3
    ws = L.sles_plan_workspace_bytes(h)
    assert ws >= 9 * lay.hc_elems * 8  # nine half-complex slots for the LES pipeline
    # compute calls without a workspace are refused, not run
    assert L.sles_fft_r2c(h, ctypes.c_void_p(16), ctypes.c_void_p(16), 1, None) == 4
    assert L.sles_plan_set_workspace(h, None, 0) == 4
    assert L.sles_plan_destroy(h) == 0


@pytest.mark.parametrize("bad,code", [
    (dict(dim=4), 1), (dict(n=100), 2), (dict(dtype=7), 1), (dict(les_model=9), 1),
    (dict(scheme=5), 1), (dict(parity=3), 1), (dict(nu=-1.0), 1), (dict(dim=3, n=1024), 2),
])
def test_plan_create_rejects(bad, code):
    L = nat.load_library()
    h = ctypes.c_void_p()
    d = _desc(**bad)
    assert L.sles_plan_create(ctypes.byref(d), ctypes.byref(h)) == code
    assert not h.value


def test_status_strings():
    L = nat.load_library()
    for s in range(8):
        assert L.sles_status_string(s)
    assert L.sles_version() == 1


def test_product_path_has_no_cpu_fallback(monkeypatch):
    import torch
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        nat.Plan(3, 32, torch.float64, 0, 0, True, 0.01, 0.1, 0.0, "cuda")
