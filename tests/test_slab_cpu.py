"""Slab decomposition on CPU: two gloo ranks advance one 3D domain split in
ky rows / x planes (sles.slab.SlabDomain, the reference's PFFT slab layout,
src/initialize_domain.py:59-65) through the two all-to-all exchanges of every
RHS evaluation, with a torch stand-in for the slab kernels
(tests/slab_cpu_backend.py).  After two reference RK3 steps the gathered
field equals the one-rank plain torch.fft path to round-off (1e-12 relative),
the ranks agree on u_max (all-reduced, src/SM_solver.py:245-255), and one
rank's slab equals its rows of the whole field.
"""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _field(n, seed=3):
    from oracle import spectral_oracle as so
    u = so.random_spectrum_velocity(n, k0=3.0, u0=1.0, seed=seed)
    return torch.fft.rfftn(torch.as_tensor(__import__("numpy").array(u)), dim=(1, 2, 3))


def _worker(rank, world, port, n, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    for p in (here, os.path.dirname(here), os.path.join(os.path.dirname(here), "spectral-les_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from slab_cpu_backend import CpuSlabPlan
        from sles.plain_torch import PlainSolver
        from sles.slab import SlabDomain
        Uh = _field(n)
        sd = SlabDomain(n, nu=1e-3, dt=2e-3, method="RK3", les="Smagorinsky", Cs=0.17, dtype=torch.float64,
                        nranks=world, rank=rank, device="cpu", plan_factory=CpuSlabPlan)
        sd.set_state(Uh)
        ps = PlainSolver(n, 3, nu=1e-3, dt=2e-3, les="Smagorinsky", Cs=0.17, method="RK3", parity=True,
                         dtype=torch.float64, device="cpu")
        ref = Uh.clone()
        umax_ref = []
        for _ in range(2):
            umax_ref.append(float(ps.irfft(ref).max()))
            sd.step()
            ref = ps.step(ref)
        got = sd.gather()
        err = float(torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref))
        rows = slice(rank * sd.m, (rank + 1) * sd.m)
        err_local = float(torch.linalg.vector_norm(sd.local() - ref[:, :, rows]) / torch.linalg.vector_norm(ref[:, :, rows]))
        q.put((rank, err, err_local, sd.u_max, umax_ref[-1]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_slab_rk3_two_gloo_ranks_match_one_rank(world):
    n = 16
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, err, err_local, umax, umax_ref in res:
        assert err < 1e-12, (rank, err)
        assert err_local < 1e-12, (rank, err_local)
        assert umax == pytest.approx(umax_ref, rel=1e-12)
