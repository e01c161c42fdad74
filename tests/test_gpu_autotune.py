"""Kernel variants and the autotuner: every x-pass variant gives the same
states (float32: variants 0-2 bit-identical, the TMA-ring variant 3 within
1e-6 relative, the compiler being free to contract a*b+c differently in it;
float64 up to contraction, 1e-14 relative); tune() picks one, records it and
new domains pick it up.  Variant 3 is compiled for the 3D grids 128, 256 and
512 (elsewhere it runs variant 0)."""
import json

import pytest
import torch

from sles import autotune, RK3_method, RK4_method, ETD2_method
from sles import _native as nat
from sles.initial import initial_velocity, initial_vorticity
from sles.initialize_domain import InitializeDomain
from sles.synthetic import gaussian_vorticity_2d, random_spectrum_velocity

pytestmark = pytest.mark.gpu

STEP = {"RK3": RK3_method.solveForNextTimestep, "RK4": RK4_method.solveForNextTimestep,
        "ETD2": ETD2_method.solveForNextTimestep}
CASES = [  # (dim, n, dtype, les, method, parity)
    (3, 64, "float32", "Smagorinsky", "RK3", True),
    (3, 96, "float32", "vreman", "RK4", True),
    (3, 128, "float32", "Smagorinsky", "ETD2", False),
    (3, 48, "float64", "Smagorinsky", "RK4", True),
    (3, 64, "float32", None, "RK4", True),
    (2, 256, "float32", None, "RK4", True),
    (3, 128, "float32", "Smagorinsky", "RK3", True),
    (3, 128, "float64", "vreman", "RK4", True),
    (3, 128, "float32", None, "RK4", True),
    (3, 128, "float64", "Smagorinsky", "ETD2", True),
    (3, 256, "float32", "Smagorinsky", "RK3", True),
    (3, 256, "float32", "Smagorinsky", "RK3", False),
]
NV = 4


def _dom(dim, n, dtype, les, method, parity):
    d = InitializeDomain(nu=1e-3, dimension=dim, time_stepSize=1e-3, No_of_gridpoint=(4 if les else 1) * n,
                         method=method, LES_ON=1 if les else 0, LES_model=les, Cs=0.17, dtype=dtype,
                         parity_mode=parity)
    if dim == 3:
        initial_velocity(d, *random_spectrum_velocity(n, 4.0, 1.0, seed=2))
    else:
        initial_vorticity(d, gaussian_vorticity_2d(n, seed=2))
    d.U_hat1[...] = d.U_hat
    return d


@pytest.mark.parametrize("case", CASES, ids=lambda c: "%dd%d_%s_%s_%s" % (c[0], c[1], c[2], c[3], c[4]))
def test_variants_are_bit_identical(case):
    ref = None
    for v in range(NV):
        d = _dom(*case)
        assert d._plan.variant_count(nat.PASS_X) == NV
        d._plan.set_variant(v, nat.PASS_X)
        for _ in range(3):
            STEP[case[4]](d)
        d._plan.check()
        u = d.U_hat.clone()
        del d
        if ref is None:
            ref = u
        elif case[2] == "float32" and v < 3:
            assert torch.equal(u, ref), "x-pass variant %d differs" % v
        elif case[2] == "float32":
            rel = float(torch.linalg.vector_norm(u - ref) / torch.linalg.vector_norm(ref))
            assert rel < 1e-6, "x-pass variant %d differs by %g" % (v, rel)
        else:
            rel = float(torch.linalg.vector_norm(u - ref) / torch.linalg.vector_norm(ref))
            assert rel < 1e-14, "x-pass variant %d differs by %g" % (v, rel)


def test_tune_records_and_reapplies(tmp_path, monkeypatch):
    monkeypatch.setenv("SLES_TUNE_CACHE", str(tmp_path / "tune.json"))
    d = _dom(3, 64, "float32", "Smagorinsky", "RK3", True)
    before = d.U_hat.clone()
    report = autotune.tune(d, steps=2, repeats=2)
    times = report[nat.PASS_X]
    assert set(times) == set(range(NV)) and all(t > 0 for t in times.values())
    win = min(times, key=times.get)
    assert d._plan.get_variant(nat.PASS_X) == win
    assert torch.equal(d.U_hat, before)  # tuning does not advance the domain
    table = json.loads((tmp_path / "tune.json").read_text())
    key = autotune.plan_key(d._plan, "RK3")
    assert table[key]["variants"][str(nat.PASS_X)] == win
    d2 = _dom(3, 64, "float32", "Smagorinsky", "RK3", True)
    assert d2._plan.get_variant(nat.PASS_X) == win
    # stepping after tuning matches an untuned domain
    d3 = _dom(3, 64, "float32", "Smagorinsky", "RK3", True)
    for _ in range(2):
        RK3_method.solveForNextTimestep(d)
        RK3_method.solveForNextTimestep(d3)
    assert torch.equal(d.U_hat, d3.U_hat)


@pytest.mark.parametrize("n,les,method", [(128, "Smagorinsky", "RK3"), (256, "Smagorinsky", "RK3"),
                                          (128, None, "RK4")])
def test_y_and_z_variants_agree_and_are_tuned(n, les, method, tmp_path, monkeypatch):
    """The y-pass tile widths and the z-pass lines per item give the same
    states (float32 bit-identical: the same arithmetic per line), and tune()
    records a choice for every pass with variants."""
    ref = None
    for py, pz in ((0, 0), (1, 0), (0, 1), (1, 1)):
        d = _dom(3, n, "float32", les, method, True)
        assert d._plan.variant_count(nat.PASS_Y) == 2 and d._plan.variant_count(nat.PASS_Z) == 2
        d._plan.set_variant(py, nat.PASS_Y)
        d._plan.set_variant(pz, nat.PASS_Z)
        for _ in range(2):
            STEP[method](d)
        d._plan.check()
        u = d.U_hat.clone()
        if ref is None:
            ref = u
        else:
            assert torch.equal(u, ref), "y/z variants (%d, %d) differ" % (py, pz)
    monkeypatch.setenv("SLES_TUNE_CACHE", str(tmp_path / "tune.json"))
    report = autotune.tune(d, steps=1, repeats=1)
    assert set(report) == {nat.PASS_X, nat.PASS_Y, nat.PASS_Z}
    table = json.loads((tmp_path / "tune.json").read_text())
    ent = table[autotune.plan_key(d._plan, method)]["variants"]
    assert {int(k) for k in ent} == {nat.PASS_X, nat.PASS_Y, nat.PASS_Z}
