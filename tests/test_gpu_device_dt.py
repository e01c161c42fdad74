"""spectralMethodSolver with the time-step logic on the GPU (device_dt=True)
takes the same steps, dt and E(k) snapshots as the host loop."""
import pytest
import torch

from sles.SM_solver import spectralMethodSolver
from sles.initial import initial_velocity
from sles.initialize_domain import InitializeDomain
from sles.synthetic import random_spectrum_velocity, taylor_green

pytestmark = pytest.mark.gpu

CASES = [  # n, dtype, les, method, parity, final time (5 to 20 steps)
    (32, "float64", None, "RK4", True, 0.8),
    (48, "float64", "Smagorinsky", "RK3", True, 0.2),
    (32, "float64", "vreman", "ETD2", False, 0.3),
    (64, "float32", "Smagorinsky", "RK4", True, 0.12),
]


def _dom(n, dtype, les, method, parity, T):
    d = InitializeDomain(nu=2e-3, final_time=T, dimension=3, time_stepSize=1e-3, No_of_gridpoint=(4 if les else 1) * n,
                         method=method, LES_ON=1 if les else 0, LES_model=les, Cs=0.17, CFL=0.5, dtype=dtype,
                         parity_mode=parity)
    u, v, w = taylor_green(n) if les is None else random_spectrum_velocity(n, 3.0, 1.0, seed=4)
    initial_velocity(d, u, v, w)
    return d


@pytest.mark.parametrize("case", CASES, ids=lambda c: "%d_%s_%s_%s" % (c[0], c[1], c[2], c[3]))
def test_device_dt_loop_matches_host_loop(case, tmp_path, monkeypatch):
    tol = 1e-12 if case[1] == "float64" else 1e-5
    (tmp_path / "host").mkdir()
    (tmp_path / "dev").mkdir()
    a, b = _dom(*case), _dom(*case)
    monkeypatch.chdir(tmp_path / "host")
    na = spectralMethodSolver(a, No_Ek_plot=3, verbose=False)
    monkeypatch.chdir(tmp_path / "dev")
    nb = spectralMethodSolver(b, No_Ek_plot=3, verbose=False, device_dt=True, chunk=4)
    assert na == nb and na > 4
    assert abs(a.dt - b.dt) <= tol * a.dt
    rel = float(torch.linalg.vector_norm(a.U_hat - b.U_hat) / torch.linalg.vector_norm(a.U_hat))
    assert rel < tol
    ha = (tmp_path / "host" / "Ek_plot_data.csv").read_text().splitlines()
    hb = (tmp_path / "dev" / "Ek_plot_data.csv").read_text().splitlines()
    assert ha[0] == hb[0] or case[1] == "float32"   # snapshot times in the column names
    assert len(ha) == len(hb)


def test_field_dumps_match_between_loops(tmp_path, monkeypatch):
    """file_out_time: the same dumps (names and contents) from both loops."""
    import numpy as np
    case = (32, "float64", "Smagorinsky", "RK3", True, 0.3)
    for sub, dev in (("host", False), ("dev", True)):
        (tmp_path / sub).mkdir()
        monkeypatch.chdir(tmp_path / sub)
        d = _dom(*case)
        spectralMethodSolver(d, file_out_time=0.1, No_Ek_plot=2, verbose=False, device_dt=dev, chunk=4)
    names = sorted(p.name for p in (tmp_path / "host" / "dumpfile").iterdir())
    assert names == sorted(p.name for p in (tmp_path / "dev" / "dumpfile").iterdir())
    assert len([n for n in names if n.endswith(".xdmf")]) >= 3
    for n in names:
        if n.endswith(".raw"):
            a = np.fromfile(tmp_path / "host" / "dumpfile" / n)
            b = np.fromfile(tmp_path / "dev" / "dumpfile" / n)
            assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(a)
